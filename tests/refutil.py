"""Helpers shared by the parity tests: scene tensors, the reference checker
module and parsers of the reference's opaque state buffers.

The reference's buffer layouts (raster_state.cu:46-117) carve each array at
the next 128-byte-aligned address; torch CUDA allocations are at least
512-byte aligned, so offsets from the buffer start follow from the sizes.
"""
import os

import numpy as np
import pytest
import torch

from conftest import ROOT


def align128(x):
    return (x + 127) // 128 * 128


def ref_module():
    """The reference backend compiled by oracle/build_ref.py (skip if absent)."""
    import build_ref
    try:
        return build_ref.load()
    except ImportError as e:
        pytest.skip(f"reference checker not built: {e}")


def ref_geom_arrays(geom, P):
    o_nd = 0
    o_scan = align128(o_nd + 4 * P)
    o_bb = align128(o_scan + 4 * P)
    o_q = align128(o_bb + 8 * P)
    g = geom
    ndup = g[o_nd:o_nd + 4 * P].view(torch.int32)
    bbox = g[o_bb:o_bb + 8 * P].view(torch.int32).view(P, 2)
    quad = g[o_q:o_q + 4 * P].view(torch.int32)
    return ndup, bbox, quad


def ref_binning_sorted(binning, R):
    o_ku = 0
    o_k = align128(o_ku + 8 * R)
    o_vu = align128(o_k + 8 * R)
    o_v = align128(o_vu + 4 * R)
    keys = binning[o_k:o_k + 8 * R].view(torch.int64)
    vals = binning[o_v:o_v + 4 * R].view(torch.int32)
    return keys, vals


class SceneTensors:
    """Device tensors of a synthetic scene plus per-camera tensors."""

    def __init__(self, scene, device="cuda"):
        self.scene = scene
        self.dev = device
        t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dt)
        self.octpath = t(scene.octpath.reshape(-1, 1), torch.int64)
        self.octlevel = t(scene.octlevel.reshape(-1, 1), torch.int8)
        self.centers = t(scene.centers)
        self.lengths = t(scene.lengths)
        self.geos = t(scene.geos)
        self.sh0 = t(scene.sh0)
        self.shs = t(scene.shs)

    def cam(self, i):
        c = self.scene.cameras[i]
        w2c = torch.from_numpy(c.w2c).to(self.dev)
        c2w = torch.from_numpy(c.c2w).to(self.dev)
        return c, w2c, c2w


def rel_err(a, b):
    a = a.double()
    b = b.double()
    den = b.norm().item()
    return (a - b).norm().item() / max(den, 1e-30)


def sh_rgbs(C, cam_pos, deg=3):
    """Per-voxel colours of every voxel from the native SH kernel."""
    from sv_raster_b200 import _C as mC
    return mC.sh_compute(deg, torch.empty(0, dtype=torch.int64), C.centers, cam_pos, C.sh0, C.shs)


def run_view(mod, C, cam_i, ns, depth=False, dist=False, normal=False, maxw=False, bg=0.0, rgbs=None, geos=None):
    """Projection + forward of one camera through `mod` (the native `_C` ops or
    the reference module: same signatures, binding.cpp:24-55)."""
    cam, w2c, c2w = C.cam(cam_i)
    ndup, geom = mod.rasterize_preprocess(cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w,
                                          cam.near, C.octpath, C.centers, C.lengths, False)
    if rgbs is None:
        rgbs = sh_rgbs(C, c2w[:3, 3])
    geos = C.geos if geos is None else geos
    out = mod.rasterize_voxels(ns, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, bg,
                               depth, dist, normal, maxw, C.octpath, C.centers, C.lengths, geos, rgbs, geom, False)
    return dict(ndup=ndup, geom=geom, R=out[0], binning=out[1], img=out[2], color=out[3], depth=out[4],
                normal=out[5], T=out[6], max_w=out[7], rgbs=rgbs, geos=geos, cam=cam, w2c=w2c, c2w=c2w)


def run_bwd(mod, C, r, ns, dC, dT, dD=None, dN=None, depth=False, normal=False, lam_R=0.0, gt=None, lam_asc=0.0,
            lam_dist=0.0, bg=0.0):
    """Backward of a run_view result through `mod`: (dL_dgeos, dL_drgbs, subdiv_p_bw)."""
    cam = r["cam"]
    e = torch.empty(0, device="cuda")
    return mod.rasterize_voxels_backward(
        r["R"], ns, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, r["w2c"], r["c2w"], bg,
        C.octpath, C.centers, C.lengths, r["geos"], r["rgbs"], r["geom"], r["binning"], r["img"], r["T"], dC,
        dD if dD is not None else e, dN if dN is not None else e, dT, lam_R, gt if gt is not None else e, lam_asc,
        lam_dist, depth, normal, r["depth"], r["normal"], False)
