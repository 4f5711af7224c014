"""CPU tests of the oracle (no GPU).

1. The oracle is pinned against golden vectors produced by the reference CUDA
   backend itself (tests/golden/*.npz, made by tests/golden/make_golden.py):
   projection and binning integers bit-exact, compositing and gradients within
   stated tolerances (the oracle's fp32 mimic cannot reproduce CUDA's expf
   bit for bit, so a tiny fraction of early-termination decisions may differ).
2. Closed-form cases: one voxel of constant density, checked against
   alpha = 1 - exp(-100 (b - a) exp_linear_11(d)) evaluated independently.
3. The FP64 oracle's backward against central finite differences of its own
   forward (the recompute-transmittance gradient is correct).
4. Generator invariants (octree encoding round trip, no overlapping cells).
"""
import glob
import math
import os

import numpy as np
import pytest

import oracle as O
from conftest import ROOT
from sv_raster_b200 import synthetic

GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))


@pytest.fixture(scope="module")
def c1():
    return synthetic.config_scene("c1")


def test_golden_inputs_unchanged(c1):
    import make_golden
    for path in GOLDEN:
        g = np.load(path)
        assert str(g["input_digest"]) == make_golden.input_digest(c1), "synthetic generator drifted"


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_goldens(c1, path):
    g = np.load(path)
    cam = c1.cameras[int(g["camera"])]
    ns = int(g["n_samp"])
    depth, dist, normal, maxw = [bool(x) for x in g["flags"]]
    bg = float(g["bg"])
    lR, lA, lD = [float(x) for x in g["lambdas"]]
    # projection: bit-exact
    ndup, bbox, quad = O.preprocess(cam, c1.centers, c1.lengths)
    assert np.array_equal(ndup.view(np.int32), g["n_dup"])
    vis = g["visible"]
    assert np.array_equal(np.where(ndup > 0)[0], vis)
    assert np.array_equal(bbox[vis].view(np.int32), g["bbox"])
    assert np.array_equal(quad[vis].view(np.int32), g["quad"])
    # binning: bit-exact
    keys, vals, ranges = O.binning(cam, c1.octpath, ndup, bbox, quad)
    assert len(vals) == int(g["num_rendered"])
    assert np.array_equal(keys.view(np.int64), g["keys"])
    assert np.array_equal(vals.view(np.int32), g["vals"])
    assert np.array_equal(ranges.reshape(g["ranges"].shape).view(np.int32), g["ranges"])
    # SH colours of the visible voxels
    rgbs = O.sh_fwd(3, vis, c1.centers, cam.position, c1.sh0, c1.shs)
    assert np.abs(rgbs[vis] - g["rgbs"][vis]).max() < 2e-6
    rgbs = g["rgbs"]  # composite the reference's own colours
    out = O.render_fwd(cam, ranges, vals, bbox, c1.centers, c1.lengths, c1.geos, rgbs, n_samp=ns, bg=bg,
                       need_depth=depth, need_dist=dist, need_normal=normal, track_max_w=maxw)
    nc_mismatch = float((out["n_contrib"].view(np.int32) != g["n_contrib"]).mean())
    assert nc_mismatch < 2e-3, f"n_contrib mismatch fraction {nc_mismatch}"
    # fp32 accumulation error of the reference itself is ~1e-5 here (the FP64
    # oracle differs from it by that much): 5e-5 absolute on colour and T
    assert np.abs(out["color"] - g["color"]).max() < 5e-5
    assert np.abs(out["T"] - g["T"][0]).max() < 5e-5
    if depth or dist:
        assert np.abs(out["depth"] - g["depth"]).max() < 2e-4
    if normal:
        assert np.abs(out["normal"] - g["normal"]).max() < 2e-4
    if maxw:
        assert np.abs(out["max_w"] - g["max_w"][:, 0]).max() < 2e-5
    # backward on the reference's own forward state, same upstream gradient
    import make_golden
    up = make_golden.upstream(int(g["camera"]), cam.height, cam.width)
    b = O.render_bwd(cam, ranges, g["tile_last"].reshape(-1), vals, bbox, c1.centers, c1.lengths, c1.geos, rgbs,
                     g["n_contrib"].astype(np.uint32), g["T"][0], up["dC"], up["dT"][0], n_samp=ns, bg=bg,
                     dL_ddepth=up["dD"] if depth else None, dL_dnormal=up["dN"] if normal else None, lambda_R=lR,
                     gt=up["gt"] if lR > 0 else None, lambda_asc=lA, lambda_dist=lD,
                     out_depth=g["depth"] if dist else None, need_depth=depth, need_normal=normal)
    for mine, name in ((b["dL_dgeos"], "dL_dgeos"), (b["dL_drgbs"], "dL_drgbs"), (b["subdiv"], "subdiv")):
        ref = g[name].reshape(mine.shape)
        rel = np.linalg.norm(mine - ref) / max(np.linalg.norm(ref), 1e-30)
        assert rel < 1e-4, f"{name}: relative error {rel:.2e}"


def _one_voxel_scene(d, size=0.25, rgb=(0.2, 0.5, 0.9)):
    path = np.array([0], np.int64)
    centers = np.zeros((1, 3), np.float32)
    lengths = np.full((1, 1), size, np.float32)
    geos = np.full((1, 8), d, np.float32)
    rgbs = np.array([rgb], np.float32)
    return path, centers, lengths, geos, rgbs


@pytest.mark.parametrize("d", [-1.0, 0.5, 2.0])
def test_closed_form_single_voxel(d):
    cam = synthetic.make_camera(48, 40, 40.0, (0.0, 0.0, -1.2))
    path, centers, lengths, geos, rgbs = _one_voxel_scene(d)
    out = O.render_view(cam, path, centers, lengths, geos, rgbs, mode="f64", bg=0.25)
    # the rasterizer receives camera scalars and constants as fp32 (as the reference's binding does)
    d32 = float(np.float32(d))
    a32, b32 = float(np.float32(0.909090909091)), float(np.float32(0.904689820196))
    act = d32 if d32 > float(np.float32(1.1)) else math.exp(a32 * d32 - b32)
    c2w = cam.c2w.astype(np.float64)
    tfx, tfy = float(np.float32(cam.tanfovx)), float(np.float32(cam.tanfovy))
    cx, cy = float(np.float32(cam.cx)), float(np.float32(cam.cy))
    for py in range(cam.height):
        for px in range(cam.width):
            rd = np.array([(px + 0.5 - cx) * 2 * tfx / cam.width,
                           (py + 0.5 - cy) * 2 * tfy / cam.height, 1.0])
            rd = c2w[:3, :3] @ rd
            rd /= np.linalg.norm(rd)
            o = c2w[:3, 3]
            with np.errstate(divide="ignore"):
                t0 = (-0.125 - o) / rd
                t1 = (0.125 - o) / rd
            a = np.max(np.minimum(t0, t1))
            b = np.min(np.maximum(t0, t1))
            expect_T = 1.0
            if a <= b:
                alpha = min(float(np.float32(0.99999)), 1 - math.exp(-100.0 * (b - a) * act))
                if alpha >= float(np.float32(1e-5)):
                    expect_T = 1 - alpha
            ec = (1 - expect_T) * np.array(rgbs[0], np.float64) + expect_T * 0.25
            assert abs(out["T"][py, px] - expect_T) < 1e-9
            assert np.abs(out["color"][:, py, px] - ec).max() < 1e-9


def _loss(cam, sc, geos, rgbs, wC, wT):
    o = O.render_view(cam, sc["path"], sc["centers"], sc["lengths"], geos, rgbs, mode="f64")
    return float((o["color"] * wC).sum() + (o["T"] * wT).sum()), o


def test_fp64_backward_matches_finite_differences():
    """Central differences in FP64 on voxels whose colour is not clamped and
    whose alpha is not saturated (the reference backward ignores both clamps)."""
    sc0 = synthetic.config_scene("c1", n_voxels=1500)
    cam = synthetic.make_camera(40, 32, 50.0, (0.2, -0.1, -1.2))
    rng = np.random.default_rng(0)
    sc = dict(path=sc0.octpath, centers=sc0.centers, lengths=sc0.lengths)
    geos = sc0.geos.astype(np.float64)
    geos = (geos * 0.5 + 1.0)  # denser: more voxels reach visible alpha
    rgbs = rng.uniform(0.1, 0.9, size=(sc0.n_voxels, 3))
    wC = rng.standard_normal((3, cam.height, cam.width))
    wT = rng.standard_normal((cam.height, cam.width))
    L0, o = _loss(cam, sc, geos.astype(np.float32), rgbs.astype(np.float32), wC, wT)
    b = O.render_bwd(cam, o["ranges"], o["tile_last"], o["vals"], o["bbox"], sc0.centers, sc0.lengths,
                     geos.astype(np.float32), rgbs.astype(np.float32), o["n_contrib"], o["T"], wC, wT, mode="f64")
    hit = np.where(np.abs(b["dL_dgeos"]).sum(1) > 1e-6)[0]
    assert len(hit) > 20
    pick = rng.choice(hit, size=min(40, len(hit)), replace=False)
    eps = 1e-4
    num, ana = [], []
    for v in pick:
        c = int(rng.integers(0, 8))
        gp = geos.copy(); gp[v, c] += eps
        gm = geos.copy(); gm[v, c] -= eps
        # the oracle's inputs are fp32 arrays: perturb in fp32-representable steps
        Lp, _ = _loss(cam, sc, gp.astype(np.float32), rgbs.astype(np.float32), wC, wT)
        Lm, _ = _loss(cam, sc, gm.astype(np.float32), rgbs.astype(np.float32), wC, wT)
        step = float(gp[v, c].astype(np.float32)) - float(gm[v, c].astype(np.float32))
        num.append((Lp - Lm) / step)
        ana.append(b["dL_dgeos"][v, c])
        k = int(rng.integers(0, 3))
        rp = rgbs.copy(); rp[v, k] += eps
        rm = rgbs.copy(); rm[v, k] -= eps
        Lp, _ = _loss(cam, sc, geos.astype(np.float32), rp.astype(np.float32), wC, wT)
        Lm, _ = _loss(cam, sc, geos.astype(np.float32), rm.astype(np.float32), wC, wT)
        step = float(rp[v, k].astype(np.float32)) - float(rm[v, k].astype(np.float32))
        num.append((Lp - Lm) / step)
        ana.append(b["dL_drgbs"][v, k])
    num, ana = np.array(num), np.array(ana)
    rel = np.linalg.norm(num - ana) / np.linalg.norm(num)
    assert rel < 1e-3, f"FD relative error {rel:.2e}"


def test_sh_oracle_against_numpy():
    rng = np.random.default_rng(3)
    P = 50
    centers = rng.uniform(-0.5, 0.5, (P, 3)).astype(np.float32)
    sh0 = rng.normal(0, 0.3, (P, 3)).astype(np.float32)
    shs = rng.normal(0, 0.3, (P, 15, 3)).astype(np.float32)
    cam = np.array([0.3, -1.2, 0.4], np.float32)
    got = O.sh_fwd(3, np.arange(P), centers, cam, sh0, shs, mode="f64")
    d = centers.astype(np.float64) - cam
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    C1, C2 = 0.4886025119029199, [1.0925484305920792, -1.0925484305920792, 0.31539156525252005,
                                  -1.0925484305920792, 0.5462742152960396]
    C3 = [-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
          1.445305721320277, -0.5900435899266435]
    basis = [-C1 * y, C1 * z, -C1 * x, C2[0] * x * y, C2[1] * y * z, C2[2] * (2 * z * z - x * x - y * y),
             C2[3] * x * z, C2[4] * (x * x - y * y), C3[0] * y * (3 * x * x - y * y), C3[1] * x * y * z,
             C3[2] * y * (4 * z * z - x * x - y * y), C3[3] * z * (2 * z * z - 3 * x * x - 3 * y * y),
             C3[4] * x * (4 * z * z - x * x - y * y), C3[5] * z * (x * x - y * y), C3[6] * x * (x * x - 3 * y * y)]
    sh0d, shsd = sh0.astype(np.float64), shs.astype(np.float64)
    want = 0.28209479177387814 * sh0d + sum(b[:, None] * shsd[:, k] for k, b in enumerate(basis)) + 0.5
    want = np.maximum(want, 0)
    assert np.abs(got - want).max() < 1e-12


def test_adam_oracle_against_formula():
    rng = np.random.default_rng(4)
    n = 1000
    p, g = rng.standard_normal(n), rng.standard_normal(n).astype(np.float32)
    g[::5] = 0
    m, v = np.zeros(n), np.zeros(n)
    pp, mm, vv = O.adam(p, g, m, v, 1, 0.01, 0.9, 0.999, 1e-8, sparse=True, mode="f64")
    b1, b2 = np.float64(np.float32(0.9)), np.float64(np.float32(0.999))
    gm = g.astype(np.float64)
    m1 = (1 - b1) * gm
    v1 = (1 - b2) * gm * gm
    step = np.float64(np.float32(0.01 / (1 - 0.9)))
    rb = np.float64(np.float32(1 / math.sqrt(1 - 0.999)))
    want = p - step * m1 / (np.sqrt(v1) * rb + np.float64(np.float32(1e-8)))
    keep = g != 0
    assert np.allclose(pp[keep], want[keep], rtol=1e-12, atol=1e-15)
    assert np.array_equal(pp[~keep], p[~keep])


def test_generator_invariants(c1):
    ijk = synthetic.octpath_to_ijk(c1.octpath, c1.octlevel)
    assert np.array_equal(synthetic.ijk_to_octpath(ijk, c1.octlevel), c1.octpath)
    assert len(synthetic.remove_overlaps(ijk, c1.octlevel.astype(np.int64))) == c1.n_voxels
    assert c1.octlevel.min() >= 6 and c1.octlevel.max() <= 8
    lv = c1.octlevel.astype(np.int64)
    shift = 3 * (16 - lv)
    assert np.all((c1.octpath & ((np.int64(1) << shift) - 1)) == 0)  # no digits below the level
    c, s = synthetic.decode_voxels(c1.octpath, c1.octlevel)
    assert np.allclose(c, c1.centers) and np.allclose(s, c1.lengths)
    assert np.all(np.abs(c) + 0.5 * s <= 0.5 + 1e-7)


def test_binning_is_a_stable_key_sort(c1):
    cam = c1.cameras[2]
    ndup, bbox, quad = O.preprocess(cam, c1.centers, c1.lengths)
    keys, vals, ranges = O.binning(cam, c1.octpath, ndup, bbox, quad)
    assert len(keys) == int(ndup.sum())
    assert np.all(keys[1:] >= keys[:-1])
    tiles = (keys >> np.uint64(48)).astype(np.int64)
    for t in np.unique(tiles)[:50]:
        lo, hi = ranges[t]
        assert np.all(tiles[lo:hi] == t)
    # multi-quadrant voxels appear once per (quadrant, tile)
    vid = vals & 0x1FFFFFFF
    assert np.array_equal(np.bincount(vid, minlength=c1.n_voxels), ndup)


def test_sampled_tile_oracle_equals_whole_view():
    """The FP64 accuracy oracle on a seeded sample of tile runs reproduces the
    whole-view FP64 oracle on those tiles (image, T), and its backward equals
    the whole-view backward of the masked upstream gradient."""
    import accuracy
    sc = synthetic.config_scene("c1", n_voxels=4000)
    cam = sc.cameras[1]
    runs = accuracy.tile_runs(cam, n_runs=6, run_len=4, seed=3)
    assert len(runs) == 6 and all(hi - lo == 4 for lo, hi in runs)
    assert all(b[0] >= a[1] for a, b in zip(runs, runs[1:]))  # disjoint, sorted
    orc = accuracy.OracleView(sc, cam, runs)
    m = orc.mask
    assert m.sum() == 6 * 4 * 256
    rgbs = O.sh_fwd(3, orc.vis, sc.centers, cam.position, sc.sh0, sc.shs, mode="f64")
    full = O.render_view(cam, sc.octpath, sc.centers, sc.lengths, sc.geos, rgbs, mode="f64")
    assert np.array_equal(orc.color[:, m], full["color"][:, m])
    assert np.array_equal(orc.T[m], full["T"][m])
    dC = np.random.default_rng(4).standard_normal((3, cam.height, cam.width)).astype(np.float32) * 1e-3
    dgeo, dsh0, dshs = orc.backward(dC)
    dCm = np.where(m[None], dC, 0).astype(np.float32)
    g = O.render_bwd(cam, full["ranges"], full["tile_last"], full["vals"], full["bbox"], sc.centers, sc.lengths,
                     sc.geos, rgbs, full["n_contrib"], full["T"], dCm, np.zeros((cam.height, cam.width), np.float32),
                     mode="f64")
    assert np.allclose(dgeo, g["dL_dgeos"], rtol=1e-12, atol=1e-18)
    d0, _ = O.sh_bwd(3, 16, orc.vis, sc.centers, cam.position, g["dL_drgbs"], mode="f64")
    assert np.allclose(dsh0, d0, rtol=1e-12, atol=1e-18)
    rep = accuracy.report(orc, np.zeros((3, cam.height, cam.width), np.float32), {"same": full["color"]}, {}, dC)
    assert rep["same"]["image_max_abs_err"] == 0.0 and rep["same"]["psnr_delta_db"] == 0.0
