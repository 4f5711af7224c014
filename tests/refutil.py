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
