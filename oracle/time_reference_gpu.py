"""Time the reference CUDA backend (oracle/_ref) on the same GPU -- the GPU
comparator for the benchmark.  TEST / MEASUREMENT INFRASTRUCTURE ONLY.

Per view it runs the reference's own call sequence (renderer.py:66-127 and
sparse_voxel_gears/renderer.py:35-94): rasterize_preprocess, the visible-index
host sync, sh_compute, rasterize_voxels (which reads the instance count back),
an L2-loss gradient, rasterize_voxels_backward and sh_compute_bw.  Prints one
JSON line with ms/view (CUDA events around all views of a step, fp32).

With --ops it instead times the reference's grid-point gathers, TV gradient
and the plain forward / backward with depth, normal and distortion outputs on
the 2M-voxel single-view scene, with the same inputs, keys and CUDA-event
medians as ``python opbench.py`` (one JSON object).

Usage: python oracle/time_reference_gpu.py [--config c4] [--steps 3] [--warmup 1] [--ops]
"""
import argparse
import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="c4")
    ap.add_argument("--voxels", type=int, default=None)
    ap.add_argument("--views", type=int, default=None)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--ops", action="store_true", help="time the gather / TV / regulariser-output ops instead")
    a = ap.parse_args()
    if a.ops:
        return time_ops(a.voxels)
    from sv_raster_b200 import synthetic
    sc = synthetic.cached_config_scene(a.config, n_voxels=a.voxels)
    cams = sc.cameras[: a.views] if a.views else sc.cameras
    rs = ReferenceSteps(sc, cams)
    ms, inst = rs.time(a.steps, a.warmup)
    print(json.dumps({"impl": "reference-cuda-backend", "config": a.config, "voxels": sc.n_voxels,
                      "views": len(cams), "size": [cams[0].width, cams[0].height], "ms_per_view": round(ms, 3),
                      "instances_per_view": inst, "dtype": "f32", "device": torch.cuda.get_device_name()}))


class ReferenceSteps:
    """The reference backend's per-view training call sequence over a set of
    cameras (fp32 parameters, L2 loss against seeded targets)."""

    def __init__(self, sc, cams, dev="cuda"):
        import build_ref
        self.ref = build_ref.load()
        t = lambda x, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(x)).to(dev, dt)
        self.octpath, self.centers, self.lengths = (t(sc.octpath.reshape(-1, 1), torch.int64), t(sc.centers),
                                                    t(sc.lengths))
        self.geos, self.sh0, self.shs = t(sc.geos), t(sc.sh0), t(sc.shs)
        self.mats = [(c, t(c.w2c), t(c.c2w)) for c in cams]
        rng = np.random.default_rng(0)
        self.targets = [t(rng.uniform(0, 1, (3, c.height, c.width)).astype(np.float32)) for c in cams]
        self.e = torch.empty(0, device=dev)

    def view(self, i):
        ref, e = self.ref, self.e
        cam, w2c, c2w = self.mats[i]
        W, H = cam.width, cam.height
        ndup, geom = ref.rasterize_preprocess(W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, cam.near,
                                              self.octpath, self.centers, self.lengths, False)
        vis = torch.where(ndup > 0)[0]
        pos = c2w[:3, 3].contiguous()
        rgbs = ref.sh_compute(3, vis, self.centers, pos, self.sh0, self.shs)
        out = ref.rasterize_voxels(1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0, False, False,
                                   False, False, self.octpath, self.centers, self.lengths, self.geos, rgbs, geom, False)
        color, T = out[3], out[6]
        dC = (2.0 / color.numel()) * (color - self.targets[i])
        g = ref.rasterize_voxels_backward(out[0], 1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0,
                                          self.octpath, self.centers, self.lengths, self.geos, rgbs, geom, out[1],
                                          out[2], T, dC, e, e, torch.zeros_like(T), 0.0, e, 0.0, 0.0, False, False,
                                          out[4], out[5], False)
        ref.sh_compute_bw(3, 16, vis, self.centers, pos, rgbs, g[1])
        return out[0]

    def step(self):
        return sum(self.view(i) for i in range(len(self.mats)))

    def time(self, steps, warmup):
        """(device ms per view over `steps` steps after `warmup`, instances per view)."""
        for _ in range(warmup):
            self.step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        inst = 0
        for _ in range(steps):
            inst += self.step()
        e1.record()
        torch.cuda.synchronize()
        n = steps * len(self.mats)
        return e0.elapsed_time(e1) / n, inst // n


def time_ops(n_voxels, reps=10, warmup=3):
    """The reference's counterparts of the opbench operators, same inputs."""
    import build_ref
    import opbench
    from sv_raster_b200 import synthetic
    ref = build_ref.load()
    dev = torch.device("cuda")
    sc = synthetic.cached_config_scene("c2", n_voxels=n_voxels)
    N = len(sc.octpath)
    key, M = synthetic.grid_keys(sc.octpath, sc.octlevel, dev)
    care = torch.arange(N, device=dev)
    g = torch.Generator(device=dev).manual_seed(0)
    pts1 = torch.randn(M, 1, device=dev, generator=g)
    pts3 = torch.randn(M, 3, device=dev, generator=g)
    d_geo = torch.randn(N, 8, device=dev, generator=g)
    d_feat = torch.randn(N, 8, 3, device=dev, generator=g)
    sinv = torch.rand(N, device=dev, generator=g) * 100
    tv_grad = torch.zeros(M, 1, device=dev)
    tv_grad_sp = torch.where(torch.rand(M, 1, device=dev, generator=g) < 0.2, 1.0, 0.0)
    tm = lambda fn: round(opbench.time_ms(fn, reps, warmup), 4)
    ops = {
        "gather_geo": tm(lambda: ref.gather_triinterp_geo_params(key, care, pts1)),
        "gather_geo_bw": tm(lambda: ref.gather_triinterp_geo_params_bw(key, care, M, d_geo)),
        "gather_feat": tm(lambda: ref.gather_triinterp_feat_params(key, care, pts3)),
        "gather_feat_bw": tm(lambda: ref.gather_triinterp_feat_params_bw(key, care, M, d_feat)),
        "tv_bw": tm(lambda: ref.total_variation_bw(pts1, key, 0.1, sinv, False, False, tv_grad)),
        "tv_bw_sparse": tm(lambda: ref.total_variation_bw(pts1, key, 0.1, sinv, False, True, tv_grad_sp)),
    }
    cam = sc.cameras[0]
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev, torch.float32)
    octpath = torch.from_numpy(sc.octpath.reshape(-1, 1)).to(dev)
    centers, lengths, geos = t(sc.centers), t(sc.lengths), t(sc.geos)
    w2c, c2w = t(cam.w2c), t(cam.c2w)
    W, H = cam.width, cam.height
    e = torch.empty(0, device=dev)
    ndup, geom = ref.rasterize_preprocess(W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, cam.near,
                                          octpath, centers, lengths, False)
    vis = torch.where(ndup > 0)[0]
    rgbs = ref.sh_compute(3, vis, centers, c2w[:3, 3].contiguous(), t(sc.sh0), t(sc.shs))
    for label, (dep, dist, nrm) in {"plain": (False, False, False), "depth_normal": (True, False, True),
                                    "depth_normal_dist": (True, True, True)}.items():
        fwd = lambda: ref.rasterize_voxels(1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0, dep,
                                           dist, nrm, False, octpath, centers, lengths, geos, rgbs, geom, False)
        ops[f"render_fwd_{label}"] = tm(fwd)
        R, binning, img, color, depth, normal, T, _ = fwd()
        dC = torch.randn(color.shape, device=dev, generator=g) * 1e-3
        dD = torch.randn(depth.shape, device=dev, generator=g) * 1e-3 if dep else e
        dN = torch.randn(normal.shape, device=dev, generator=g) * 1e-3 if nrm else e
        dT = torch.zeros_like(T)
        bwd = lambda: ref.rasterize_voxels_backward(
            R, 1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0, octpath, centers, lengths, geos,
            rgbs, geom, binning, img, T, dC, dD, dN, dT, 0.0, color, 0.0, 0.1 if dist else 0.0, dep, nrm,
            depth, normal, False)
        ops[f"render_bwd_{label}"] = tm(bwd)
    print(json.dumps({"impl": "reference-cuda-backend", "scene": f"c2 synthetic, {N} voxels, {M} grid points",
                      "ms": ops, "device": torch.cuda.get_device_name()}))


if __name__ == "__main__":
    main()
