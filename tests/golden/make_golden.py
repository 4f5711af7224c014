"""Generate golden vectors from the reference CUDA backend (run on a GPU box).

Runs the reference's own native ops -- the module compiled from
backends/cuda by oracle/build_ref.py -- on the seeded synthetic c1 scene
(sv_raster_b200.synthetic.config_scene("c1")) and stores, per case, the
reference's outputs as compressed .npz files next to this script:

  preprocess : n_duplicates, packed bboxes and quadrant bitsets (visible rows)
  binning    : instance count, sorted keys and values, tile ranges
  forward    : tile_last, n_contrib, colour, T (+ depth / normal / max_w)
  backward   : dL_dgeos, dL_drgbs, subdiv_p_bw for a seeded upstream gradient
  sh         : the SH colours fed to the rasterizer

Inputs are not stored (they are regenerated from the seed); an input digest
is stored so a drift of the generator is detected.  Usage:
    python tests/golden/make_golden.py [out_dir]
"""
import hashlib
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

CASES = {
    # name: (camera, n_samp, depth, distortion, normal, max_w, bg, lambda_R, lambda_asc, lambda_dist)
    "c1_cam0_ns1": (0, 1, False, False, False, False, 0.0, 0.0, 0.0, 0.0),
    "c1_cam1_ns2_depth": (1, 2, True, False, False, True, 0.0, 0.0, 0.01, 0.0),
    "c1_cam2_ns3_all": (2, 3, True, True, True, True, 1.0, 0.01, 0.01, 0.1),
}


def input_digest(sc):
    h = hashlib.sha256()
    for a in (sc.octpath, sc.centers, sc.lengths, sc.geos, sc.sh0, sc.shs):
        h.update(np.ascontiguousarray(a).tobytes())
    for c in sc.cameras:
        h.update(np.ascontiguousarray(c.w2c).tobytes())
    return h.hexdigest()


def upstream(cam_i, H, W):
    rng = np.random.default_rng(100 + cam_i)
    return dict(dC=(rng.standard_normal((3, H, W)) * 1e-3).astype(np.float32),
                dT=(rng.standard_normal((1, H, W)) * 1e-3).astype(np.float32),
                dD=(rng.standard_normal((3, H, W)) * 1e-3).astype(np.float32),
                dN=(rng.standard_normal((3, H, W)) * 1e-3).astype(np.float32),
                gt=rng.uniform(0, 1, (3, H, W)).astype(np.float32))


def main(out_dir=HERE):
    import build_ref
    from refutil import ref_binning_sorted, ref_geom_arrays
    from sv_raster_b200 import synthetic
    ref = build_ref.load()
    sc = synthetic.config_scene("c1")
    dev = "cuda"
    t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)
    octpath, centers, lengths = t(sc.octpath.reshape(-1, 1), torch.int64), t(sc.centers), t(sc.lengths)
    geos, sh0, shs = t(sc.geos), t(sc.sh0), t(sc.shs)
    P = sc.n_voxels
    digest = input_digest(sc)
    for name, (ci, ns, depth, dist, normal, maxw, bg, lR, lA, lD) in CASES.items():
        cam = sc.cameras[ci]
        w2c, c2w = t(cam.w2c), t(cam.c2w)
        W, H = cam.width, cam.height
        ndup, geom = ref.rasterize_preprocess(W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, cam.near,
                                              octpath, centers, lengths, False)
        vis = torch.where(ndup > 0)[0]
        rgbs = ref.sh_compute(3, vis, centers, c2w[:3, 3].contiguous(), sh0, shs)
        out = ref.rasterize_voxels(ns, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, bg, depth, dist,
                                   normal, maxw, octpath, centers, lengths, geos, rgbs, geom, False)
        R, binning, img = out[0], out[1], out[2]
        color, odepth, onormal, T, max_w = out[3], out[4], out[5], out[6], out[7]
        nd, bb, qd = ref_geom_arrays(geom, P)
        keys, vals = ref_binning_sorted(binning, R)
        ranges, tile_last, n_contrib = ref.unpack_ImageState(W, H, img)
        up = upstream(ci, H, W)
        e = torch.empty(0, device=dev)
        g = ref.rasterize_voxels_backward(
            R, ns, W, H, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, bg, octpath, centers, lengths, geos,
            rgbs, geom, binning, img, T, t(up["dC"]), t(up["dD"]) if depth else e, t(up["dN"]) if normal else e,
            t(up["dT"]), lR, t(up["gt"]) if lR > 0 else e, lA, lD, depth, normal, odepth, onormal, False)
        torch.cuda.synchronize()
        visn = vis.cpu().numpy()
        rec = dict(
            input_digest=np.array(digest), camera=np.array(ci), n_samp=np.array(ns),
            flags=np.array([depth, dist, normal, maxw], dtype=np.int8), bg=np.array(bg, np.float32),
            lambdas=np.array([lR, lA, lD], np.float32),
            n_dup=nd.cpu().numpy(), visible=visn, bbox=bb[vis].cpu().numpy(), quad=qd[vis].cpu().numpy(),
            num_rendered=np.array(R), keys=keys.cpu().numpy(), vals=vals.cpu().numpy(),
            ranges=ranges.cpu().numpy(), tile_last=tile_last.cpu().numpy(), n_contrib=n_contrib.cpu().numpy(),
            rgbs=rgbs.cpu().numpy(), color=color.cpu().numpy(), T=T.cpu().numpy(),
            dL_dgeos=g[0].cpu().numpy(), dL_drgbs=g[1].cpu().numpy(), subdiv=g[2].cpu().numpy())
        if depth or dist:
            rec["depth"] = odepth.cpu().numpy()
        if normal:
            rec["normal"] = onormal.cpu().numpy()
        if maxw:
            rec["max_w"] = max_w.cpu().numpy()
        path = os.path.join(out_dir, f"{name}.npz")
        np.savez_compressed(path, **rec)
        print(name, "R =", R, "->", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
