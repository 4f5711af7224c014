"""CPU check of the batched path's tight pixel bbox on the oracle (no GPU).

The batched projection may replace the reference's rounded pixel bbox
(preprocess.cu:98-113: each side of the projected corners' extent rounded to
the nearest pixel) by the pixels whose centre lies within 0.05 pixel of the
unrounded extent, for voxels with all 8 corners in front of the near plane.
The claim that makes this safe: every pixel it drops has a centre ray that
misses the cube.  Here the tight bbox is restated in numpy (float64), fed to
the oracle's binning and compositing, and the images, T and gradients must be
the rounded bbox's bit for bit, with fewer instances.
"""
import numpy as np
import pytest

import oracle as O
from sv_raster_b200 import synthetic

MARGIN = 0.05


def tight_bbox(cam, centers, lengths, ndup, bbox, quad, tile=O.TILE):
    """Tight bbox, duplicate count and quadrants from the rounded ones."""
    signs = np.array([[(i >> 2) & 1, (i >> 1) & 1, i & 1] for i in range(8)], np.float64) * 2 - 1
    corners = centers[:, None, :].astype(np.float64) + 0.5 * lengths.reshape(-1, 1, 1) * signs[None]
    w2c = np.asarray(cam.w2c, np.float64)
    pc = corners @ w2c[:3, :3].T + w2c[:3, 3]
    front = (pc[..., 2] >= cam.near).all(axis=1)
    z = np.where(pc[..., 2] > 0, pc[..., 2], 1.0)
    u, v = pc[..., 0] / z, pc[..., 1] / z
    fx = 0.5 * cam.width / cam.tanfovx
    fy = 0.5 * cam.height / cam.tanfovy
    bx0 = np.maximum(fx * u.min(1) + cam.cx - 0.5, 0.0)
    by0 = np.maximum(fy * v.min(1) + cam.cy - 0.5, 0.0)
    bx1 = np.minimum(fx * u.max(1) + cam.cx - 0.5, cam.width)
    by1 = np.minimum(fy * v.max(1) + cam.cy - 0.5, cam.height)
    rx0, ry0 = (bbox[:, 0] >> 16).astype(np.int64), (bbox[:, 0] & 0xFFFF).astype(np.int64)
    rx1, ry1 = (bbox[:, 1] >> 16).astype(np.int64), (bbox[:, 1] & 0xFFFF).astype(np.int64)
    x0 = np.maximum(rx0, np.ceil(bx0 - MARGIN).astype(np.int64))
    y0 = np.maximum(ry0, np.ceil(by0 - MARGIN).astype(np.int64))
    x1 = np.minimum(rx1, np.floor(bx1 + MARGIN).astype(np.int64))
    y1 = np.minimum(ry1, np.floor(by1 + MARGIN).astype(np.int64))
    sel = (ndup > 0) & front
    empty = sel & ((x0 > x1) | (y0 > y1))
    keep = sel & ~empty
    nb, nd, nq = bbox.copy(), ndup.copy(), quad.copy()
    nb[keep, 0] = ((x0[keep] << 16) | y0[keep]).astype(np.uint32)
    nb[keep, 1] = ((x1[keep] << 16) | y1[keep]).astype(np.uint32)
    gx, gy = (cam.width + tile - 1) // tile, (cam.height + tile - 1) // tile
    tx0 = np.clip(x0 // tile, 0, gx - 1)
    ty0 = np.clip(y0 // tile, 0, gy - 1)
    tx1 = np.clip(x1 // tile, 0, gx - 1)
    ty1 = np.clip(y1 // tile, 0, gy - 1)
    pop = np.array([bin(int(q)).count("1") for q in quad], np.int64)
    nd[keep] = ((tx1 - tx0 + 1) * (ty1 - ty0 + 1) * pop)[keep].astype(np.uint32)
    nd[empty], nq[empty] = 0, 0
    nb[empty] = 0
    return nd, nb, nq


@pytest.fixture(scope="module")
def c1():
    return synthetic.config_scene("c1")


@pytest.mark.parametrize("cam_i", [0, 2])
def test_tight_bbox_drops_only_missing_rays(c1, cam_i):
    cam = c1.cameras[cam_i]
    ndup, bbox, quad = O.preprocess(cam, c1.centers, c1.lengths)
    tnd, tbb, tq = tight_bbox(cam, c1.centers, c1.lengths, ndup, bbox, quad)
    assert (tnd <= ndup).all()
    vis = np.where(ndup > 0)[0]
    rgbs = O.sh_fwd(3, vis, c1.centers, cam.position, c1.sh0, c1.shs)
    outs = []
    for nd, bb, q in ((ndup, bbox, quad), (tnd, tbb, tq)):
        keys, vals, ranges = O.binning(cam, c1.octpath, nd, bb, q)
        o = O.render_fwd(cam, ranges, vals, bb, c1.centers, c1.lengths, c1.geos, rgbs)
        rng = np.random.default_rng(3)
        dC = rng.standard_normal(o["color"].shape).astype(np.float32)
        dT = rng.standard_normal(o["T"].shape).astype(np.float32)
        g = O.render_bwd(cam, ranges, o["tile_last"], vals, bb, c1.centers, c1.lengths, c1.geos, rgbs,
                         o["n_contrib"], o["T"], dC, dT)
        outs.append((len(vals), o, g))
    (n_r, o_r, g_r), (n_t, o_t, g_t) = outs
    print(f"camera {cam_i}: {n_t} of {n_r} instances with the tight bbox ({1 - n_t / n_r:.1%} dropped)")
    assert n_t < n_r
    assert np.array_equal(o_t["color"], o_r["color"])
    assert np.array_equal(o_t["T"], o_r["T"])
    assert (o_t["n_contrib"] <= o_r["n_contrib"]).all()
    for k in g_r:
        if isinstance(g_r[k], np.ndarray) and g_r[k].dtype.kind == "f":
            scale = max(float(np.abs(g_r[k]).max()), 1e-30)
            assert float(np.abs(g_t[k] - g_r[k]).max()) <= 1e-6 * scale, k
