"""GPU parity of the native path against the reference backend and the oracle.

Bit-exact: duplicate counts, packed bboxes, quadrant bitsets, instance count,
sorted keys and values, tile ranges, tile_last and per-pixel contributor
counts.  Within tolerance (stated per check): images, transmittance, depth,
normal, max_w and the gradients (whose atomic summation order is not fixed in
either implementation).
"""
import numpy as np
import pytest
import torch

import oracle as O
from refutil import (SceneTensors, ref_binning_sorted, ref_geom_arrays, ref_module, rel_err, run_bwd, run_view,
                     sh_rgbs)
from sv_raster_b200 import _C as mC
from sv_raster_b200 import synthetic

pytestmark = pytest.mark.gpu

# Gradients are sums of many per-pixel terms accumulated with atomics in an
# order that differs between the two implementations: tolerance is norm-wise.
GRAD_REL_TOL = 1e-5
IMG_ABS_TOL = 1e-5


@pytest.fixture(scope="module")
def c1():
    return SceneTensors(synthetic.config_scene("c1"))


@pytest.fixture(scope="module")
def ref():
    return ref_module()


def _rgbs(C, cam_pos, deg=3):
    return sh_rgbs(C, cam_pos, deg)


_run = run_view
_bwd = run_bwd


CASES = [
    # (camera, n_samp, depth, distortion, normal, max_w, bg)
    (0, 1, False, False, False, False, 0.0),
    (1, 1, False, False, False, True, 1.0),
    (2, 1, True, True, True, True, 0.0),
    (0, 2, True, False, False, False, 0.0),
    (2, 3, True, False, True, False, 1.0),
    (1, 3, False, True, False, False, 0.0),
]


@pytest.mark.parametrize("cam_i,ns,depth,dist,normal,maxw,bg", CASES)
def test_forward_bit_exact_integers(c1, ref, cam_i, ns, depth, dist, normal, maxw, bg):
    P = c1.centers.shape[0]
    a = _run(mC, c1, cam_i, ns, depth, dist, normal, maxw, bg)
    b = _run(ref, c1, cam_i, ns, depth, dist, normal, maxw, bg, rgbs=a["rgbs"])
    torch.cuda.synchronize()
    # preprocess
    assert torch.equal(a["ndup"], b["ndup"])
    nd, bb, qd, = mC.unpack_geom_state(a["geom"], P)[0], mC.unpack_geom_state(a["geom"], P)[2], \
        mC.unpack_geom_state(a["geom"], P)[3]
    rnd, rbb, rqd = ref_geom_arrays(b["geom"], P)
    vis = rnd > 0
    assert torch.equal(nd, rnd)
    assert torch.equal(bb[vis], rbb[vis])
    assert torch.equal(qd[vis], rqd[vis])
    # binning
    assert a["R"] == b["R"]
    R = a["R"]
    k, v = mC.unpack_sorted_list(a["binning"], R, a["cam"].width, a["cam"].height)
    rk, rv = ref_binning_sorted(b["binning"], R)
    assert torch.equal(v, rv), "sorted values differ"
    assert torch.equal(k, rk), "sorted keys differ"
    ra, ta, na = mC.unpack_ImageState(a["cam"].width, a["cam"].height, a["img"])
    rr, rt, rn = ref.unpack_ImageState(a["cam"].width, a["cam"].height, b["img"])
    assert torch.equal(ra, rr), "tile ranges differ"
    assert torch.equal(ta, rt), "tile_last differs"
    assert torch.equal(na, rn), "n_contrib differs"
    # floating outputs
    assert (a["color"] - b["color"]).abs().max().item() <= IMG_ABS_TOL
    assert (a["T"] - b["T"]).abs().max().item() <= IMG_ABS_TOL
    if depth or dist:
        assert (a["depth"] - b["depth"]).abs().max().item() <= 1e-4
    if normal:
        assert (a["normal"] - b["normal"]).abs().max().item() <= IMG_ABS_TOL
    if maxw:
        assert (a["max_w"] - b["max_w"]).abs().max().item() <= IMG_ABS_TOL


def test_forward_images_bitwise_identical(c1, ref):
    """Same arithmetic as the reference: the default image is bit-identical."""
    a = _run(mC, c1, 0, 1)
    b = _run(ref, c1, 0, 1, rgbs=a["rgbs"])
    assert torch.equal(a["color"], b["color"])
    assert torch.equal(a["T"], b["T"])


@pytest.mark.parametrize("cam_i,ns,depth,dist,normal,maxw,bg", CASES)
def test_backward_matches_reference(c1, ref, cam_i, ns, depth, dist, normal, maxw, bg):
    a = _run(mC, c1, cam_i, ns, depth, dist, normal, maxw, bg)
    b = _run(ref, c1, cam_i, ns, depth, dist, normal, maxw, bg, rgbs=a["rgbs"])
    cam = a["cam"]
    g = torch.Generator(device="cuda").manual_seed(cam_i * 10 + ns)
    H, W = cam.height, cam.width
    dC = torch.randn(3, H, W, device="cuda", generator=g) * 1e-3
    dT = torch.randn(1, H, W, device="cuda", generator=g) * 1e-3
    dD = torch.randn(3, H, W, device="cuda", generator=g) * 1e-3 if depth else None
    dN = torch.randn(3, H, W, device="cuda", generator=g) * 1e-3 if normal else None
    gt = torch.rand(3, H, W, device="cuda", generator=g)
    kw = dict(depth=depth, normal=normal, lam_R=0.01 if cam_i == 2 else 0.0, gt=gt, lam_asc=0.01 if ns > 1 else 0.0,
              lam_dist=0.1 if dist else 0.0, bg=bg)
    ga = _bwd(mC, c1, a, ns, dC, dT, dD, dN, **kw)
    gb = _bwd(ref, c1, b, ns, dC, dT, dD, dN, **kw)
    for x, y, name in zip(ga, gb, ("dL_dgeos", "dL_drgbs", "subdiv_p_bw")):
        assert x.shape == y.shape, name
        e = rel_err(x, y)
        assert e <= GRAD_REL_TOL, f"{name}: relative error {e:.3e}"


def test_against_cpu_oracle(c1):
    """GPU fp32 vs the oracle's fp32 mimic and fp64 modes on every c1 camera."""
    for cam_i in range(3):
        a = _run(mC, c1, cam_i, 1)
        sc = c1.scene
        cam = sc.cameras[cam_i]
        rgbs = a["rgbs"].cpu().numpy()
        o32 = O.render_view(cam, sc.octpath, sc.centers, sc.lengths, sc.geos, rgbs, mode="f32")
        o64 = O.render_view(cam, sc.octpath, sc.centers, sc.lengths, sc.geos, rgbs, mode="f64")
        col = a["color"].cpu().numpy()
        assert np.abs(col - o32["color"]).max() < 1e-4
        assert np.abs(col - o64["color"]).max() < 1e-4
        nc = mC.unpack_ImageState(cam.width, cam.height, a["img"])[2].cpu().numpy()
        mism = (nc != o32["n_contrib"]).mean()
        assert mism < 1e-3, f"n_contrib mismatch fraction {mism}"
        k, v = mC.unpack_sorted_list(a["binning"], a["R"], cam.width, cam.height)
        assert np.array_equal(v.cpu().numpy().view(np.uint32), o32["vals"])
        assert np.array_equal(k.cpu().numpy().view(np.uint64), o32["keys"])


def test_sh_matches_reference(c1, ref):
    cam, w2c, c2w = c1.cam(1)
    pos = c2w[:3, 3].contiguous()
    idx = torch.arange(0, c1.centers.shape[0], 3, device="cuda")
    for deg in range(4):
        shs = c1.shs[:, : (deg + 1) ** 2 - 1].contiguous() if deg < 3 else c1.shs
        a = mC.sh_compute(deg, idx, c1.centers, pos, c1.sh0, shs)
        b = ref.sh_compute(deg, idx, c1.centers, pos, c1.sh0, shs)
        assert torch.equal(a, b)
        g = torch.randn_like(a)
        M = 1 + shs.shape[1]
        a0, a1 = mC.sh_compute_bw(deg, M, idx, c1.centers, pos, a, g)
        b0, b1 = ref.sh_compute_bw(deg, M, idx, c1.centers, pos, b, g)
        assert torch.equal(a0, b0) and torch.equal(a1, b1)


@pytest.mark.parametrize("sparse", [False, True])
def test_adam_matches_reference(ref, sparse):
    g = torch.Generator(device="cuda").manual_seed(3)
    n = 100_003
    p0 = torch.randn(n, device="cuda", generator=g)
    grad = torch.randn(n, device="cuda", generator=g)
    grad[::7] = 0
    pa, pb = p0.clone(), p0.clone()
    ma, va = torch.zeros_like(p0), torch.zeros_like(p0)
    mb, vb = torch.zeros_like(p0), torch.zeros_like(p0)
    for step in range(1, 4):
        mC.unbiased_adam_step(sparse, pa, grad, ma, va, step, 0.025, 0.1, 0.99, 1e-15)
        ref.unbiased_adam_step(sparse, pb, grad, mb, vb, step, 0.025, 0.1, 0.99, 1e-15)
    assert torch.equal(pa, pb) and torch.equal(ma, mb) and torch.equal(va, vb)
    mC.biased_adam_step(sparse, pa, grad, ma, va, 0.01, 0.9, 0.999, 1e-8)
    ref.biased_adam_step(sparse, pb, grad, mb, vb, 0.01, 0.9, 0.999, 1e-8)
    assert torch.equal(pa, pb) and torch.equal(ma, mb) and torch.equal(va, vb)


def test_gather_matches_reference(ref):
    g = torch.Generator(device="cuda").manual_seed(5)
    M, N = 5000, 2000
    key = torch.randint(0, M, (N, 8), device="cuda", generator=g)
    care = torch.randperm(N, device="cuda", generator=g)[:1500]
    pts = torch.randn(M, 1, device="cuda", generator=g)
    a = mC.gather_triinterp_geo_params(key, care, pts)
    b = ref.gather_triinterp_geo_params(key, care, pts)
    assert torch.equal(a[care], b[care])
    d = torch.randn(N, 8, device="cuda", generator=g)
    ga = mC.gather_triinterp_geo_params_bw(key, care, M, d)
    gb = ref.gather_triinterp_geo_params_bw(key, care, M, d)
    assert rel_err(ga, gb) < 1e-6
    f = torch.randn(M, 3, device="cuda", generator=g)
    assert torch.equal(mC.gather_triinterp_feat_params(key, care, f)[care],
                       ref.gather_triinterp_feat_params(key, care, f)[care])


def test_empty_scene_and_empty_view(c1):
    """P = 0, and a camera that sees nothing: outputs are background."""
    cam, w2c, c2w = c1.cam(0)
    e3 = torch.zeros(0, 3, device="cuda")
    nd, geom = mC.rasterize_preprocess(64, 48, cam.tanfovx, cam.tanfovy, 32, 24, w2c, c2w, 0.02,
                                       torch.zeros(0, 1, dtype=torch.int64, device="cuda"), e3,
                                       torch.zeros(0, 1, device="cuda"))
    assert nd.numel() == 0
    # camera outside the scene looking away from it
    away = synthetic.make_camera(64, 48, 50.0, (0.0, 0.0, -1.5), target=(0.0, 0.0, -3.0))
    w2c_away = torch.from_numpy(away.w2c).cuda()
    c2w_away = torch.from_numpy(away.c2w).cuda()
    rg = torch.rand(c1.centers.shape[0], 3, device="cuda")
    nd, geom = mC.rasterize_preprocess(64, 48, cam.tanfovx, cam.tanfovy, 32, 24, w2c_away, c2w_away, 0.02,
                                       c1.octpath, c1.centers, c1.lengths)
    assert int(nd.sum()) == 0
    out = mC.rasterize_voxels(1, 64, 48, cam.tanfovx, cam.tanfovy, 32, 24, w2c_away, c2w_away, 0.5, False, False,
                              False, False, c1.octpath, c1.centers, c1.lengths, c1.geos, rg, geom)
    assert out[0] == 0
    assert torch.all(out[3] == 0.5) and torch.all(out[6] == 1.0)


@pytest.mark.parametrize("no_tv_s", [False, True])
def test_total_variation_matches_reference_dense(ref, no_tv_s):
    from sv_raster_b200 import grid_loss_bw
    g = torch.Generator(device="cuda").manual_seed(11)
    M, N = 4000, 1500
    key = torch.randint(0, M, (N, 8), device="cuda", generator=g)
    pts = torch.randn(M, 1, device="cuda", generator=g)
    sinv = torch.rand(N, device="cuda", generator=g) * 100
    a = torch.randn(M, 1, device="cuda", generator=g)
    b = a.clone()
    grid_loss_bw.total_variation(pts, key, 0.1, sinv, no_tv_s, False, a)
    ref.total_variation_bw(pts, key, 0.1, sinv, no_tv_s, False, b)
    assert rel_err(a, b) < 1e-6


@pytest.mark.parametrize("C", [1, 2, 3])
def test_total_variation_sparse_rule(C):
    """Sparse mode touches only voxels with a non-zero corner gradient, judged on
    the gradient as it was before the call (numpy statement of the rule), for
    the one- and three-channel kernels and the generic channel count."""
    from sv_raster_b200 import grid_loss_bw
    rng = np.random.default_rng(12)
    M, N = 3000, 800
    key = rng.integers(0, M, (N, 8))
    pts = rng.standard_normal((M, C)).astype(np.float32)
    grad0 = np.where(rng.uniform(size=(M, C)) < 0.2, rng.standard_normal((M, C)), 0).astype(np.float32)
    sinv = rng.uniform(1, 50, N).astype(np.float32)
    want = grad0.astype(np.float64).copy()
    for n in range(N):
        for c in range(C):
            k = key[n]
            if not np.any(grad0[k, c] != 0):
                continue
            v = pts[k, c]
            w = 0.5 * 0.01 * sinv[n]
            for i in range(8):
                s = sum((1 if v[i] > v[i ^ m] else -1) for m in (1, 2, 4))
                want[k[i], c] += w * s
    got = torch.from_numpy(grad0).cuda()
    grid_loss_bw.total_variation(torch.from_numpy(pts).cuda(), torch.from_numpy(key).cuda(), 0.5,
                                 torch.from_numpy(sinv).cuda(), False, True, got)
    assert np.abs(got.cpu().numpy() - want).max() < 1e-4
