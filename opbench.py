"""Device timings of the plain-path operators around the core render step.

Run on a GPU as ``python opbench.py [--voxels N]``; prints one
JSON object.  Every figure is the median of CUDA-event timings on the current
stream after warm-up, on the seeded 2M-voxel scene with one 1297x840 view
(the single-view benchmark scene):

* ``gather_geo`` / ``gather_geo_bw`` / ``gather_feat`` / ``gather_feat_bw`` --
  grid-point gathers of geo_params_gather.cu (the voxels' 8 corners index a
  deduplicated grid of corner points), forward and backward, all voxels cared
  for.  HBM roofline with the algorithmic bytes given beside each entry.
* ``tv_bw`` / ``tv_bw_sparse`` -- total-variation gradient on the grid points
  (tv_compute.cu), dense and sparse.
* ``render_*`` -- forward and backward compositing of the view with depth,
  distortion and normal outputs off and on (the regulariser inputs of
  backward.cu), showing what the extra outputs cost on top of the colour.

``--grid-step c2,c4`` instead times the batched step with grid-point
densities, gathered and scattered separately or fused into the compositing
kernels (see ``grid_step``).

Inputs of the gathers are larger than L2 (126 MB) only for their index
arrays; the grid values themselves are read at random, so their figures are
bounded by the gather pattern rather than by streaming bandwidth.
"""
import argparse
import json
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from sv_raster_b200 import _C as mC  # noqa: E402
from sv_raster_b200 import synthetic  # noqa: E402
from sv_raster_b200.grid_loss_bw import total_variation  # noqa: E402
from sv_raster_b200.synthetic import grid_keys  # noqa: E402


def time_ms(fn, reps, warmup):
    for _ in range(warmup):
        fn()
    st = torch.cuda.current_stream()
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    out.sort()
    return out[len(out) // 2]


def _peak_gbs():
    here = os.path.dirname(os.path.abspath(__file__))
    try:
        with open(os.path.join(here, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


class _DevCam:
    def __init__(self, c, dev):
        self.width, self.height, self.tanfovx, self.tanfovy = c.width, c.height, c.tanfovx, c.tanfovy
        self.cx, self.cy, self.near = c.cx, c.cy, c.near
        self.w2c = torch.from_numpy(c.w2c).to(dev)
        self.c2w = torch.from_numpy(c.c2w).to(dev)


def grid_step(configs, reps, warmup):
    """Batched compositing of a configuration's views with grid-point
    densities, two ways: the separate all-voxel gather + render + backward +
    scatter, and the fused form whose staging reads the grid points and whose
    flush adds into the grid gradient (svr_batch_render_grid /
    svr_batch_backward_grid).  8x8 tiles, forward staging 64, backward
    staging 32 with two pixels per thread, fp32 grid; prepare excluded."""
    from sv_raster_b200.batched import BatchedRasterizer, gather_grid_geos, scatter_grid_grad
    dev = torch.device("cuda")
    t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)
    out = {}
    for name in configs:
        sc = synthetic.cached_config_scene(name)
        key, grid_np = synthetic.grid_params(sc, dev)
        key, grid = key.contiguous(), t(grid_np)
        P, M = sc.n_voxels, grid.numel()
        r = BatchedRasterizer([_DevCam(c, dev) for c in sc.cameras], t(sc.octpath.reshape(-1), torch.int64),
                              t(sc.centers), t(sc.lengths), max_level=sc.max_level, tile_size=8)
        r.set_staging(64)
        r.set_backward_staging(32)
        r.set_backward_pixels_per_thread(2)
        sh0, shs = t(sc.sh0), t(sc.shs)
        r.fit_capacity(sh0, shs, 3)
        r.prepare(sh0, shs, 3)
        g = torch.Generator(device=dev).manual_seed(3)
        dC = torch.randn(3 * r.n_pixels, device=dev, generator=g) * 1e-3
        dT = torch.zeros(r.n_pixels, device=dev)
        geos, dgeos, dgrid = torch.empty(P, 8, device=dev), torch.zeros(P, 8, device=dev), torch.zeros(M, device=dev)
        color, T = torch.empty(3 * r.n_pixels, device=dev), torch.empty(r.n_pixels, device=dev)

        def separate():
            gather_grid_geos(key, grid, geos)
            r.render(geos, color, T)
            dgeos.zero_()
            r.backward_render(geos, T, dC, dT, dgeos)
            scatter_grid_grad(key, dgeos, dgrid)

        def fused():
            r.render_grid(key, grid, color, T)
            r.backward_render_grid(key, grid, T, dC, dT, dgrid)

        ops = {"separate": separate, "fused": fused,
               "gather": lambda: gather_grid_geos(key, grid, geos),
               "render": lambda: r.render(geos, color, T),
               "backward": lambda: r.backward_render(geos, T, dC, dT, dgeos),
               "scatter": lambda: scatter_grid_grad(key, dgeos, dgrid),
               "render_grid": lambda: r.render_grid(key, grid, color, T),
               "backward_grid": lambda: r.backward_render_grid(key, grid, T, dC, dT, dgrid)}
        out[name] = {"voxels": P, "grid_points": M, "views": len(sc.cameras), "instances": r.header()[0],
                     "ms": {k: round(time_ms(fn, reps, warmup), 4) for k, fn in ops.items()}}
        del r
        torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--voxels", type=int, default=None)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--grid-step", default=None,
                    help="comma-separated configurations (e.g. c2,c4): separate vs fused grid-point batched step")
    args = ap.parse_args()
    if not torch.cuda.is_available():
        raise SystemExit("opbench needs a CUDA device")
    if args.grid_step:
        res = grid_step(args.grid_step.split(","), args.reps, args.warmup)
        res["device"] = torch.cuda.get_device_name(torch.device("cuda"))
        print(json.dumps(res))
        return
    dev = torch.device("cuda")
    sc = synthetic.cached_config_scene("c2", n_voxels=args.voxels)
    N = len(sc.octpath)
    key, M = grid_keys(sc.octpath, sc.octlevel, dev)
    care = torch.arange(N, device=dev)
    g = torch.Generator(device=dev).manual_seed(0)
    pts1 = torch.randn(M, 1, device=dev, generator=g)
    pts3 = torch.randn(M, 3, device=dev, generator=g)
    d_geo = torch.randn(N, 8, device=dev, generator=g)
    d_feat = torch.randn(N, 8, 3, device=dev, generator=g)
    sinv = torch.rand(N, device=dev, generator=g) * 100
    tv_grad = torch.zeros(M, 1, device=dev)
    tv_grad_sp = torch.where(torch.rand(M, 1, device=dev, generator=g) < 0.2, 1.0, 0.0)
    peak, peak_kind = _peak_gbs()
    res = {"scene": f"c2 synthetic, {N} voxels, {M} grid points, 1 view 1297x840", "peak_gbs": peak,
           "peak_kind": peak_kind, "ops": {}}

    def hbm(name, fn, bytes_):
        ms = time_ms(fn, args.reps, args.warmup)
        gbs = bytes_ / (ms * 1e-3) / 1e9
        res["ops"][name] = {"ms": round(ms, 4), "alg_bytes": int(bytes_), "gbs": round(gbs, 1),
                            "frac": round(gbs / peak, 3)}

    # per voxel: 8 int64 keys + care index + 8 gathered values + 8 outputs (C channels)
    hbm("gather_geo", lambda: mC.gather_triinterp_geo_params(key, care, pts1), N * (64 + 8 + 32 + 32))
    hbm("gather_geo_bw", lambda: mC.gather_triinterp_geo_params_bw(key, care, M, d_geo),
        N * (64 + 8 + 32 + 32) + M * 4)
    hbm("gather_feat", lambda: mC.gather_triinterp_feat_params(key, care, pts3), N * (64 + 8 + 96 + 96))
    hbm("gather_feat_bw", lambda: mC.gather_triinterp_feat_params_bw(key, care, M, d_feat),
        N * (64 + 8 + 96 + 96) + M * 12)
    # per voxel: 8 keys + 8 grid values + 1/size + 8 gradient read-modify-writes
    hbm("tv_bw", lambda: total_variation(pts1, key, 0.1, sinv, False, False, tv_grad), N * (64 + 32 + 4 + 64))
    hbm("tv_bw_sparse", lambda: total_variation(pts1, key, 0.1, sinv, False, True, tv_grad_sp),
        N * (64 + 32 + 4 + 64))

    # forward / backward compositing with the regulariser outputs off and on
    cam = sc.cameras[0]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev, torch.float32)
    octpath = torch.from_numpy(sc.octpath.reshape(-1, 1)).to(dev)
    centers, lengths, geos = t(sc.centers), t(sc.lengths), t(sc.geos)
    w2c, c2w = t(cam.w2c), t(cam.c2w)
    W, H = cam.width, cam.height
    ndup, geom = mC.rasterize_preprocess(W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, cam.near,
                                         octpath, centers, lengths)
    vis = torch.where(ndup > 0)[0]
    rgbs = mC.sh_compute(3, vis, centers, c2w[:3, 3].contiguous(), t(sc.sh0), t(sc.shs))
    for label, (dep, dist, nrm) in {"plain": (False, False, False), "depth_normal": (True, False, True),
                                    "depth_normal_dist": (True, True, True)}.items():
        fwd = lambda: mC.rasterize_voxels(1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0, dep,
                                          dist, nrm, False, octpath, centers, lengths, geos, rgbs, geom)
        res["ops"][f"render_fwd_{label}"] = {"ms": round(time_ms(fwd, args.reps, args.warmup), 4)}
        R, binning, img, color, depth, normal, T, _ = fwd()
        dC = torch.randn(color.shape, device=dev, generator=g) * 1e-3
        dT = torch.zeros_like(T)
        dD = torch.randn(depth.shape, device=dev, generator=g) * 1e-3 if dep else torch.empty(0)
        dN = torch.randn(normal.shape, device=dev, generator=g) * 1e-3 if nrm else torch.empty(0)
        bwd = lambda: mC.rasterize_voxels_backward(
            R, 1, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0, octpath, centers, lengths, geos,
            rgbs, geom, binning, img, T, dC, dD, dN, dT, 0.0, color, 0.0, 0.1 if dist else 0.0, dep, nrm,
            depth if dist else torch.empty(0), normal if nrm else torch.empty(0))
        res["ops"][f"render_bwd_{label}"] = {"ms": round(time_ms(bwd, args.reps, args.warmup), 4)}
    res["device"] = torch.cuda.get_device_name(dev)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
