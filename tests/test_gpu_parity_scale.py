"""Reference-backend parity on the benchmark configurations at full size.

The reference backend (compiled from its own sources into oracle/_ref) and
this repository's plain path run on the same seeded inputs:

* c2: the 2M-voxel scene, its full 1297x840 view;
* c3: the same kind of scene seen by two of its 16 orbit cameras (the
  largest one and a small one);
* c4: the 8M-voxel scene (levels 8-14), one full 1920x1080 view in fp32.

Bit-exact: duplicate counts, packed bboxes and quadrant bitsets (visible
voxels), the instance count, sorted keys and values, tile ranges, tile_last
and per-pixel contributor counts.  Bitwise: images and T.  Within 1e-5
norm-wise relative error: dL_dgeos, dL_drgbs, subdiv_p_bw and the SH
gradients of an L2 loss (both sides accumulate with atomics in different
orders).  The reference code exercised is forward.cu:601-734 and
backward.cu:655-769 with the kernels they launch.

The batched multi-view path (bf16 storage, 8x8 tiles) is compared on one
c4 1080p view with the reference fed the same bf16-rounded densities and SH
coefficients upcast to fp32: colours bitwise; images bitwise with the exact
arithmetic, within 1e-5 norm-wise with the fast one; gradients within 1e-5.
"""
import numpy as np
import pytest
import torch

from refutil import (SceneTensors, ref_binning_sorted, ref_geom_arrays, ref_module, rel_err, run_bwd, run_view)
from sv_raster_b200 import _C as mC
from sv_raster_b200 import synthetic
from sv_raster_b200.batched import BatchedRasterizer

pytestmark = pytest.mark.gpu

GRAD_REL_TOL = 1e-5
IMG_TOL = 1e-5


@pytest.fixture(scope="module")
def ref():
    return ref_module()


_scenes = {}


def scene(name):
    if name not in _scenes:
        _scenes.clear()  # keep one full-size scene on the device at a time
        torch.cuda.empty_cache()
        _scenes[name] = SceneTensors(synthetic.cached_config_scene(name))
    return _scenes[name]


def c3_views():
    cams = synthetic.cached_config_scene("c3").cameras
    px = [c.width * c.height for c in cams]
    return [int(np.argmax(px)), int(np.argmin(px))]


def _integer_parity(a, b, P, ref):
    assert torch.equal(a["ndup"], b["ndup"]), "n_duplicates differ"
    nd, _, bb, qd = mC.unpack_geom_state(a["geom"], P)[:4]
    rnd, rbb, rqd = ref_geom_arrays(b["geom"], P)
    vis = rnd > 0
    assert torch.equal(nd, rnd)
    assert torch.equal(bb[vis], rbb[vis]), "packed bboxes differ"
    assert torch.equal(qd[vis], rqd[vis]), "quadrant bitsets differ"
    assert a["R"] == b["R"], f"instance count {a['R']} vs {b['R']}"
    R = a["R"]
    cam = a["cam"]
    k, v = mC.unpack_sorted_list(a["binning"], R, cam.width, cam.height)
    rk, rv = ref_binning_sorted(b["binning"], R)
    assert torch.equal(k, rk), "sorted keys differ"
    assert torch.equal(v, rv), "sorted values differ"
    ra, ta, na = mC.unpack_ImageState(cam.width, cam.height, a["img"])
    rr, rt, rn = ref.unpack_ImageState(cam.width, cam.height, b["img"])
    assert torch.equal(ra, rr), "tile ranges differ"
    assert torch.equal(ta, rt), "tile_last differs"
    assert torch.equal(na, rn), "n_contrib differs"
    return R


def _loss_grad(color, seed):
    """Gradient of an L2 loss against a seeded uniform target."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    target = torch.rand(color.shape, device="cuda", generator=g)
    return (2.0 / color.numel()) * (color - target)


@pytest.mark.parametrize("name,cam_i", [("c2", 0), ("c3", "largest"), ("c3", "smallest"), ("c4", 0)])
def test_plain_path_matches_reference_at_full_size(ref, name, cam_i):
    if cam_i in ("largest", "smallest"):
        cam_i = c3_views()[0 if cam_i == "largest" else 1]
    C = scene(name)
    P = C.centers.shape[0]
    a = run_view(mC, C, cam_i, 1)
    b = run_view(ref, C, cam_i, 1, rgbs=a["rgbs"])
    torch.cuda.synchronize()
    R = _integer_parity(a, b, P, ref)
    assert R > 0
    assert torch.equal(a["color"], b["color"]), "images differ"
    assert torch.equal(a["T"], b["T"]), "transmittance differs"
    dC = _loss_grad(a["color"], 7)
    dT = torch.zeros_like(a["T"])
    ga = run_bwd(mC, C, a, 1, dC, dT)
    gb = run_bwd(ref, C, b, 1, dC, dT)
    errs = {}
    for x, y, nm in zip(ga, gb, ("dL_dgeos", "dL_drgbs", "subdiv_p_bw")):
        assert x.shape == y.shape, nm
        errs[nm] = rel_err(x, y)
    # SH backward of each side's colour gradient (the reference's call sequence, sh_compute.cu:270-299)
    pos = a["c2w"][:3, 3].contiguous()
    vis = torch.nonzero(a["ndup"] > 0).reshape(-1)
    sa = mC.sh_compute_bw(3, 16, vis, C.centers, pos, a["rgbs"], ga[1])
    sb = ref.sh_compute_bw(3, 16, vis, C.centers, pos, b["rgbs"], gb[1])
    errs["dL_dsh0"] = rel_err(sa[0], sb[0])
    errs["dL_dshs"] = rel_err(sa[1], sb[1])
    print(f"{name} view {cam_i} ({a['cam'].width}x{a['cam'].height}, {P} voxels, {R} instances): "
          + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v <= GRAD_REL_TOL, f"{k}: relative error {v:.3e}"


class _DevCam:
    def __init__(self, c):
        self.width, self.height = c.width, c.height
        self.tanfovx, self.tanfovy, self.cx, self.cy, self.near = c.tanfovx, c.tanfovy, c.cx, c.cy, c.near
        self.w2c = torch.from_numpy(c.w2c).cuda()
        self.c2w = torch.from_numpy(c.c2w).cuda()


@pytest.mark.parametrize("exact,ppt", [(True, 1), (False, 1), (True, 2), (False, 2)])
def test_batched_bf16_c4_view_matches_reference_on_rounded_inputs(ref, exact, ppt):
    """The batched step on one 1080p c4 view (bf16 storage, 8x8 tiles) against
    the reference run on the bf16-rounded parameters upcast to fp32.  With the
    exact arithmetic images and T are bitwise the reference's; with the fast
    one (the default) within 1e-5 norm-wise, and at most ~1e-4 at a pixel
    whose transmittance lands on the early-stop threshold."""
    C = scene("c4")
    sc = C.scene
    cam = sc.cameras[0]
    geos16 = C.geos.to(torch.bfloat16).contiguous()
    sh016, shs16 = C.sh0.to(torch.bfloat16).contiguous(), C.shs.to(torch.bfloat16).contiguous()
    r = BatchedRasterizer([_DevCam(cam)], C.octpath, C.centers, C.lengths, max_level=sc.max_level, tile_size=8,
                          exact=exact)
    r.set_pixels_per_thread(ppt)
    r.fit_capacity(sh016, shs16, 3)
    r.prepare(sh016, shs16, 3)
    color, T = r.render(geos16)
    torch.cuda.synchronize()
    total, err = r.header()
    assert err == 0 and 0 < total <= r.capacity
    color = color.view(3, cam.height, cam.width)
    T = T.view(1, cam.height, cam.width)

    # the reference on the rounded parameters
    w2c, c2w = torch.from_numpy(cam.w2c).cuda(), torch.from_numpy(cam.c2w).cuda()
    pos = c2w[:3, 3].contiguous()
    geos32, sh032, shs32 = geos16.float(), sh016.float(), shs16.float()
    ndup, geom = ref.rasterize_preprocess(cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w,
                                          cam.near, C.octpath, C.centers, C.lengths, False)
    vis = torch.where(ndup > 0)[0]
    rgbs = ref.sh_compute(3, vis, C.centers, pos, sh032, shs32)
    out = ref.rasterize_voxels(1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0,
                               False, False, False, False, C.octpath, C.centers, C.lengths, geos32, rgbs, geom, False)
    rcolor, rT = out[3], out[6]
    brgbs = r.arrays()["rgbs"][0]
    # the fast arithmetic's tight pixel bbox culls a voxel whose rays all miss
    # (no colour computed); every voxel it keeps is one the reference keeps
    bvis = torch.where(r.arrays()["ndup"][0] > 0)[0]
    assert bool((ndup[bvis] > 0).all()) and (len(bvis) == len(vis) if exact else len(bvis) <= len(vis))
    rgb_bitwise = bool(torch.equal(brgbs[bvis], rgbs[bvis]))
    img_max = (color - rcolor).abs().max().item()
    img_rel = rel_err(color, rcolor)
    t_max = (T - rT).abs().max().item()
    bitwise = bool(torch.equal(color, rcolor) and torch.equal(T, rT))

    dC = _loss_grad(color, 9)
    dT = torch.zeros_like(T)
    dgeo, sub, dsh0, dshs = r.backward(geos16, T.reshape(-1), dC.reshape(-1).contiguous(), dT.reshape(-1), 3, 16)
    e = torch.empty(0, device="cuda")
    g = ref.rasterize_voxels_backward(out[0], 1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c,
                                      c2w, 0.0, C.octpath, C.centers, C.lengths, geos32, rgbs, geom, out[1], out[2],
                                      rT, dC, e, e, dT, 0.0, e, 0.0, 0.0, False, False, out[4], out[5], False)
    rsh0, rshs = ref.sh_compute_bw(3, 16, vis, C.centers, pos, rgbs, g[1])
    errs = {"dL_dgeos": rel_err(dgeo, g[0]), "subdiv_p_bw": rel_err(sub, g[2].reshape(-1)),
            "dL_dsh0": rel_err(dsh0, rsh0), "dL_dshs": rel_err(dshs, rshs)}
    print(f"batched c4 view 0 ({'exact' if exact else 'fast'}, {ppt} px/thread) vs reference (bf16-rounded inputs): rgb bitwise "
          f"{rgb_bitwise}, image max err {img_max:.2e} rel {img_rel:.2e}, T max err {t_max:.2e}, bitwise {bitwise}; "
          + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    assert rgb_bitwise
    if exact:
        assert bitwise
    else:
        assert img_rel <= IMG_TOL and img_max <= 2e-4 and rel_err(T, rT) <= IMG_TOL
    for k, v in errs.items():
        assert v <= GRAD_REL_TOL, f"{k}: relative error {v:.3e}"


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_grid_points_batched_matches_reference(ref, name):
    """Grid-point densities (the reference's training parametrisation): the
    batched step's gather -> render -> backward -> scatter against the
    reference's gather_triinterp_geo_params + rasterize + its backward +
    gather_triinterp_geo_params_bw (renderer.py:319-345,
    geo_params_gather.cu:22-72) on view 0: gathered corners and images
    bitwise (fp32, exact arithmetic), grid gradient within 1e-5."""
    from sv_raster_b200.batched import GridBatchedRender
    C = scene(name)
    sc = C.scene
    key, grid_np = synthetic.grid_params(sc, torch.device("cuda"))
    grid = torch.from_numpy(grid_np).cuda()
    cam = sc.cameras[0]
    r = BatchedRasterizer([_DevCam(cam)], C.octpath, C.centers, C.lengths, max_level=sc.max_level, tile_size=8,
                          exact=True)
    r.fit_capacity(C.sh0, C.shs, 3)
    g = grid.clone().requires_grad_(True)
    color, T = GridBatchedRender.apply(r, 3, key, g, C.sh0, C.shs)
    dC = _loss_grad(color.view(3, cam.height, cam.width), 21)
    color.backward(dC.reshape(-1))
    # the reference: gather, per-view rasterize, backward, scatter
    P = C.centers.shape[0]
    care = torch.arange(P, device="cuda")
    geos = ref.gather_triinterp_geo_params(key, care, grid.view(-1, 1))
    w2c, c2w = torch.from_numpy(cam.w2c).cuda(), torch.from_numpy(cam.c2w).cuda()
    pos = c2w[:3, 3].contiguous()
    ndup, geom = ref.rasterize_preprocess(cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w,
                                          cam.near, C.octpath, C.centers, C.lengths, False)
    vis = torch.where(ndup > 0)[0]
    rgbs = ref.sh_compute(3, vis, C.centers, pos, C.sh0, C.shs)
    out = ref.rasterize_voxels(1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0,
                               False, False, False, False, C.octpath, C.centers, C.lengths, geos, rgbs, geom, False)
    e = torch.empty(0, device="cuda")
    gr = ref.rasterize_voxels_backward(out[0], 1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy,
                                       w2c, c2w, 0.0, C.octpath, C.centers, C.lengths, geos, rgbs, geom, out[1],
                                       out[2], out[6], dC, e, e, torch.zeros_like(out[6]), 0.0, e, 0.0, 0.0, False,
                                       False, out[4], out[5], False)
    dgrid = ref.gather_triinterp_geo_params_bw(key, care, grid.numel(), gr[0]).reshape(-1)
    assert torch.equal(color.detach().view(3, cam.height, cam.width), out[3]), "images differ"
    err = rel_err(g.grad, dgrid)
    print(f"{name}: {grid.numel()} grid points, grid gradient rel err {err:.2e}")
    assert err <= GRAD_REL_TOL
