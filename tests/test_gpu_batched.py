"""GPU tests of the multi-view batched path: per view it must reproduce the
plain path (bit-identical images and contributor counts in fp32 storage
with the exact arithmetic; within fp32 accumulation error with the fast one),
gradients summed over views must match the plain per-view sums, bf16 storage
must stay within the PSNR budget of the FP64 oracle, the CUDA-graph replay
must equal eager execution, and capacity overflow must be reported, not
crash."""
import math
import os

import numpy as np
import pytest
import torch

import oracle as O
from refutil import SceneTensors, rel_err
from sv_raster_b200 import _C as mC
from sv_raster_b200 import synthetic
from sv_raster_b200.batched import BatchedRasterizer, BatchedRender

pytestmark = pytest.mark.gpu


class DevCam:
    def __init__(self, c):
        self.width, self.height = c.width, c.height
        self.tanfovx, self.tanfovy, self.cx, self.cy, self.near = c.tanfovx, c.tanfovy, c.cx, c.cy, c.near
        self.w2c = torch.from_numpy(c.w2c).cuda()
        self.c2w = torch.from_numpy(c.c2w).cuda()


@pytest.fixture(scope="module")
def c1():
    return SceneTensors(synthetic.config_scene("c1"))


def _plain_view(C, cam_i, sh0, shs, geos):
    cam, w2c, c2w = C.cam(cam_i)
    ndup, geom = mC.rasterize_preprocess(cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w,
                                         cam.near, C.octpath, C.centers, C.lengths)
    vis = torch.where(ndup > 0)[0]
    rgbs = mC.sh_compute(3, vis, C.centers, c2w[:3, 3].contiguous(), sh0, shs)
    out = mC.rasterize_voxels(1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c, c2w, 0.0,
                              False, False, False, False, C.octpath, C.centers, C.lengths, geos, rgbs, geom)
    return dict(ndup=ndup, geom=geom, R=out[0], binning=out[1], img=out[2], color=out[3], T=out[6], rgbs=rgbs,
                vis=vis, cam=cam, w2c=w2c, c2w=c2w)


def _raster(C, max_level=None, views=(0, 1, 2), **kw):
    cams = [DevCam(C.scene.cameras[i]) for i in views]
    r = BatchedRasterizer(cams, C.octpath, C.centers, C.lengths,
                          max_level=max_level or C.scene.max_level, **kw)
    return r, cams


@pytest.mark.parametrize("binning,ppt", [(1, 1), (0, 1), (1, 2)])
@pytest.mark.parametrize("max_key_bits", [None, 40])
def test_batched_forward_equals_plain(c1, max_key_bits, binning, ppt, monkeypatch):
    """Counting sort by tile (binning 1) and radix passes over the tile bits
    (0, with one or several sort groups) give the plain path's tile lists;
    with the exact arithmetic images, T and contributor counts are the plain
    path's with one or two pixels per compositing thread."""
    if max_key_bits:
        # 32 position bits + 8 bits for one view's tiles: one sort group per view
        monkeypatch.setenv("SVR_MAX_KEY_BITS", str(max_key_bits))
    r, _ = _raster(c1, exact=True)
    r.set_pixels_per_thread(ppt)
    r.set_binning(binning)
    if max_key_bits:
        assert r.n_groups == 3
    total = r.fit_capacity(c1.sh0, c1.shs, 3)
    r.prepare(c1.sh0, c1.shs, 3)
    color, T = r.render(c1.geos)
    torch.cuda.synchronize()
    n, err = r.header()
    assert err == 0 and n == total
    arr = r.arrays()
    cols, Ts = r.split_color(color), r.split_pixels(T)
    tile0 = 0
    for k in range(3):
        p = _plain_view(c1, k, c1.sh0, c1.shs, c1.geos)
        assert torch.equal(arr["ndup"][k], p["ndup"])
        assert torch.equal(arr["rgbs"][k][p["vis"]], p["rgbs"][p["vis"]])
        assert torch.equal(cols[k], p["color"]), f"view {k}: colour differs"
        assert torch.equal(Ts[k], p["T"]), f"view {k}: T differs"
        cam = p["cam"]
        pr, ptl, pnc = mC.unpack_ImageState(cam.width, cam.height, p["img"])
        H, W = cam.height, cam.width
        nc = arr["n_contrib"][r.pix_offsets[k]:r.pix_offsets[k + 1]].view(H, W)
        assert torch.equal(nc, pnc), f"view {k}: n_contrib differs"
        nt = pr.shape[0] * pr.shape[1]
        br = arr["ranges"][tile0:tile0 + nt].view(pr.shape)
        btl = arr["tile_last"][tile0:tile0 + nt].view(ptl.shape)
        assert torch.equal(br[..., 1] - br[..., 0], pr[..., 1] - pr[..., 0])
        assert torch.equal(btl - br[..., 0], ptl - pr[..., 0])
        # the tile lists themselves (values) are the plain path's, tile by tile
        _, pv = mC.unpack_sorted_list(p["binning"], p["R"], W, H)
        bv = arr["sorted_vals"]
        nz = (pr[..., 1] > pr[..., 0]).reshape(-1).nonzero().reshape(-1)
        for t in nz[:: max(1, len(nz) // 25)].tolist():
            a0, a1 = int(pr.view(-1, 2)[t, 0]), int(pr.view(-1, 2)[t, 1])
            b0 = int(br.view(-1, 2)[t, 0])
            assert torch.equal(bv[b0:b0 + a1 - a0], pv[a0:a1])
        tile0 += nt


@pytest.mark.parametrize("binning", [1, 0])
def test_large_tile_segments_match_plain_sort(binning):
    """Low-resolution views put up to ~20k instances in one 16x16 tile, so the
    per-tile segment sort takes its streamed (larger than shared memory) path
    (and the counting sort's per-tile atomics are at their most contended);
    every tile list must still equal the plain path's full-key radix sort."""
    import dataclasses
    sc = synthetic.config_scene("c1")
    cams = [synthetic.make_camera(16, 16, 70.0, (0.3, -0.4, 3.2)), synthetic.make_camera(48, 40, 60.0, (0.0, 2.0, 2.5)),
            synthetic.make_camera(64, 64, 90.0, (2.2, 0.5, -1.8))]
    C = SceneTensors(dataclasses.replace(sc, cameras=cams))
    r = BatchedRasterizer([DevCam(c) for c in cams], C.octpath, C.centers, C.lengths, max_level=sc.max_level,
                          exact=True)
    r.set_binning(binning)
    r.fit_capacity(C.sh0, C.shs, 3)
    r.prepare(C.sh0, C.shs, 3)
    color, T = r.render(C.geos)
    torch.cuda.synchronize()
    assert r.header()[1] == 0
    arr = r.arrays()
    cols = r.split_color(color)
    tile0, biggest = 0, 0
    for k in range(len(cams)):
        p = _plain_view(C, k, C.sh0, C.shs, C.geos)
        assert torch.equal(cols[k], p["color"]), f"view {k}: colour differs"
        cam = p["cam"]
        pr, _, _ = mC.unpack_ImageState(cam.width, cam.height, p["img"])
        _, pv = mC.unpack_sorted_list(p["binning"], p["R"], cam.width, cam.height)
        nt = pr.shape[0] * pr.shape[1]
        pr2 = pr.view(-1, 2)
        br2 = arr["ranges"][tile0:tile0 + nt].view(-1, 2)
        assert torch.equal(br2[:, 1] - br2[:, 0], pr2[:, 1] - pr2[:, 0])
        for t in range(nt):
            a0, a1, b0 = int(pr2[t, 0]), int(pr2[t, 1]), int(br2[t, 0])
            biggest = max(biggest, a1 - a0)
            assert torch.equal(arr["sorted_vals"][b0:b0 + a1 - a0], pv[a0:a1]), f"view {k} tile {t}"
        tile0 += nt
    assert biggest > 4096, biggest  # the streamed segment path ran


def test_batched_backward_equals_plain_sum(c1):
    r, _ = _raster(c1)
    r.fit_capacity(c1.sh0, c1.shs, 3)
    geos = c1.geos.clone().requires_grad_(True)
    sh0 = c1.sh0.clone().requires_grad_(True)
    shs = c1.shs.clone().requires_grad_(True)
    color, T = BatchedRender.apply(r, 3, geos, sh0, shs)
    g = torch.Generator(device="cuda").manual_seed(7)
    wC = torch.randn(color.shape, device="cuda", generator=g)
    wT = torch.randn(T.shape, device="cuda", generator=g)
    ((color * wC).sum() + (T * wT).sum()).backward()
    # plain path, one view at a time through the reference-compatible autograd surface
    from sv_raster_b200 import renderer
    geos2 = c1.geos.clone().requires_grad_(True)
    sh02 = c1.sh0.clone().requires_grad_(True)
    shs2 = c1.shs.clone().requires_grad_(True)
    wCs, wTs = r.split_color(wC), r.split_pixels(wT)
    for k in range(3):
        cam, w2c, c2w = c1.cam(k)
        s = renderer.RasterSettings("sh", 1, cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c,
                                    c2w)

        def vox_fn(idx, cam_pos, mode):
            rg = renderer.SH_eval.apply(3, idx, c1.centers, cam_pos, None, sh02, shs2)
            return {"geos": geos2, "rgbs": rg, "subdiv_p": torch.ones(len(c1.centers), 1, device="cuda")}

        col, _, _, Tk, _ = renderer.rasterize_voxels(s, c1.octpath, c1.centers, c1.lengths, vox_fn)
        ((col * wCs[k]).sum() + (Tk * wTs[k]).sum()).backward()
    assert rel_err(geos.grad, geos2.grad) < 1e-5
    assert rel_err(sh0.grad, sh02.grad) < 1e-5
    assert rel_err(shs.grad, shs2.grad) < 1e-5


@pytest.mark.parametrize("views", [(0, 1, 2), "c3"])
def test_fast_arithmetic_matches_exact(c1, views):
    """The default fast compositing arithmetic (hardware exponential,
    approximate division) against the exact form that is bit-identical to the
    plain path: images within 1e-5 norm-wise (a pixel whose transmittance
    lands on the early-stop threshold may take one voxel more or less, at most
    about 1e-4 of colour), contributor counts equal almost everywhere (on the
    reference's rounded bbox; the default tight bbox of the fast form shortens
    the lists, so its counts are compared by the culling test), and gradients
    within 1e-5."""
    if views == "c3":
        C = SceneTensors(synthetic.cached_config_scene("c3"))
        cams = [DevCam(C.scene.cameras[i]) for i in (0, 5)]
    else:
        C = c1
        cams = [DevCam(C.scene.cameras[i]) for i in views]
    out = {}
    g = torch.Generator(device="cuda").manual_seed(13)
    for exact, culling in ((True, -1), (False, -1), (False, 0)):
        r = BatchedRasterizer(cams, C.octpath, C.centers, C.lengths, max_level=C.scene.max_level, tile_size=8,
                              exact=exact)
        r.set_culling(culling)
        if "wC" not in out:
            out["wC"] = torch.randn(3 * r.n_pixels, device="cuda", generator=g) * 1e-3
            out["wT"] = torch.randn(r.n_pixels, device="cuda", generator=g) * 1e-3
        res = _render_and_grads(r, C, out["wC"], out["wT"])
        out[exact, culling] = res + (r.arrays()["n_contrib"].clone(),)
        del r
    e, f, f0 = out[True, -1], out[False, -1], out[False, 0]
    img_rel = rel_err(f[0], e[0])
    img_max = (f[0] - e[0]).abs().max().item()
    nc_mism = (f0[7] != e[7]).float().mean().item()
    assert f[6] < f0[6] == e[6]  # the tight bbox drops instances
    assert rel_err(f0[0], e[0]) < 1e-5
    grads = {name: rel_err(a, b) for a, b, name in zip(f[2:6], e[2:6], ("dL_dgeos", "subdiv", "dL_dsh0", "dL_dshs"))}
    print(f"fast vs exact ({views}): image rel {img_rel:.2e}, max {img_max:.2e}, n_contrib mismatch {nc_mism:.2e}, "
          + ", ".join(f"{k} {v:.2e}" for k, v in grads.items()))
    assert img_rel < 1e-5 and img_max < 2e-4
    assert rel_err(f[1], e[1]) < 1e-5
    assert nc_mism < 1e-3
    for k, v in grads.items():
        assert v < 1e-5, k


@pytest.mark.parametrize("views,tile,exact", [((0, 1, 2), 8, True), ((0, 1, 2), 8, False), ((0, 1, 2), 16, True),
                                              ("c3", 8, False)])
def test_tight_bbox_culls_only_missing_rays(c1, views, tile, exact):
    """The tight pixel bbox (pixel centres within 0.05 pixel of the projected
    corners' extent) against the reference's rounded bbox, with the same
    arithmetic: the dropped (tile, voxel) instances are ones whose rays all
    miss the cube, so images and T are bit-identical, gradients agree up to
    the order of additions, every voxel's duplicate count can only shrink,
    and each pixel's last contributor sits no later in its shorter list."""
    if views == "c3":
        C = SceneTensors(synthetic.cached_config_scene("c3"))
        cams = [DevCam(C.scene.cameras[i]) for i in (0, 5)]
    else:
        C = c1
        cams = [DevCam(C.scene.cameras[i]) for i in views]
    g = torch.Generator(device="cuda").manual_seed(19)
    out = {}
    for culling in (0, 1):
        r = BatchedRasterizer(cams, C.octpath, C.centers, C.lengths, max_level=C.scene.max_level, tile_size=tile,
                              exact=exact)
        r.set_culling(culling)
        if "wC" not in out:
            out["wC"] = torch.randn(3 * r.n_pixels, device="cuda", generator=g)
            out["wT"] = torch.randn(r.n_pixels, device="cuda", generator=g)
        res = _render_and_grads(r, C, out["wC"], out["wT"])
        arr = r.arrays()
        out[culling] = res + (arr["n_contrib"].clone(), arr["ndup"].clone())
        del r
    ref, tight = out[0], out[1]
    print(f"tight bbox ({views}, {tile}x{tile}, {'exact' if exact else 'fast'}): {tight[6]} of {ref[6]} instances "
          f"({1 - tight[6] / ref[6]:.1%} dropped)")
    assert tight[6] < ref[6]
    assert torch.equal(tight[0], ref[0]), "colour differs"
    assert torch.equal(tight[1], ref[1]), "T differs"
    for a, b, name in zip(tight[2:6], ref[2:6], ("dL_dgeos", "subdiv", "dL_dsh0", "dL_dshs")):
        assert rel_err(a, b) < 1e-5, name
    assert bool((tight[7] <= ref[7]).all())
    assert bool((tight[8] <= ref[8]).all())


def _psnr(a, b):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return 10 * math.log10(1.0 / max(mse, 1e-30))


def test_bf16_storage_psnr_vs_fp64_oracle(c1):
    """bf16 storage, fp32 compositing: the image's PSNR against a target is
    within 0.01 dB of the FP64 oracle's on the same (bf16-rounded) parameters."""
    geos16 = c1.geos.to(torch.bfloat16)
    sh016, shs16 = c1.sh0.to(torch.bfloat16), c1.shs.to(torch.bfloat16)
    r, _ = _raster(c1)
    r.fit_capacity(sh016, shs16, 3)
    r.prepare(sh016, shs16, 3)
    color, T = r.render(geos16)
    cols = r.split_color(color)
    sc = c1.scene
    g64 = geos16.float().cpu().numpy()
    for k in range(3):
        cam = sc.cameras[k]
        rgbs = O.sh_fwd(3, np.arange(sc.n_voxels), sc.centers, cam.position, sh016.float().cpu().numpy(),
                        shs16.float().cpu().numpy(), mode="f64")
        o = O.render_view(cam, sc.octpath, sc.centers, sc.lengths, g64, rgbs.astype(np.float32), mode="f64")
        tgt = np.random.default_rng(k).uniform(0, 1, size=o["color"].shape)
        ours = cols[k].cpu().numpy()
        assert abs(_psnr(ours, tgt) - _psnr(o["color"], tgt)) < 0.01
        assert np.abs(ours - o["color"]).max() < 1e-4


def test_graph_replay_equals_eager(c1):
    from sv_raster_b200.workload import BatchedWorkload
    sc = synthetic.config_scene("c1")
    sc.targets = [np.random.default_rng(1).uniform(0, 1, (3, c.height, c.width)).astype(np.float32)
                  for c in sc.cameras]
    wl = BatchedWorkload(sc, torch.device("cuda"), storage=torch.float32, tune=False)
    wl._eager_step(False)
    torch.cuda.synchronize()
    c_eager, dgeo_eager = wl.color.clone(), wl.grads[0].clone()
    wl.capture()
    wl.graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(wl.color, c_eager)
    assert rel_err(wl.grads[0], dgeo_eager) < 1e-6
    # moving a camera in place is picked up by the replay
    wl.cams[0].c2w[0, 3] += 0.01
    wl.cams[0].w2c.copy_(torch.linalg.inv(wl.cams[0].c2w))
    wl.graph.replay()
    torch.cuda.synchronize()
    assert not torch.equal(wl.color, c_eager)
    assert wl.check_errors() > 0


def test_capacity_overflow_is_reported(c1):
    r, _ = _raster(c1, capacity=1000)
    r.prepare(c1.sh0, c1.shs, 3)
    r.render(c1.geos)
    torch.cuda.synchronize()
    total, err = r.header()
    assert total > 1000
    assert err & 0x4


@pytest.mark.parametrize("binning", [1, 0])
def test_zero_capacity_renders_background(c1, binning):
    """A plan without instance capacity (before fit_capacity) reports the
    overflow and composites every tile as empty: background colour, T = 1."""
    r, _ = _raster(c1, capacity=0)
    r.set_binning(binning)
    r.prepare(c1.sh0, c1.shs, 3)
    color, T = r.render(c1.geos)
    torch.cuda.synchronize()
    total, err = r.header()
    assert total > 0 and err & 0x4
    assert torch.all(T == 1.0) and torch.all(color == 0.0)


def test_level_bound_is_checked(c1):
    r, _ = _raster(c1, max_level=5)  # the c1 voxels are at levels 6-8
    r.fit_capacity(c1.sh0, c1.shs, 3)
    r.prepare(c1.sh0, c1.shs, 3)
    torch.cuda.synchronize()
    assert r.header()[1] & 0x10


def test_training_step_graph_matches_plain_form():
    """Three training steps (fwd + bwd + Adam): the captured batched step with
    fp32 storage and the device step counter tracks the plain per-view step
    with SparseAdam."""
    from sv_raster_b200.workload import BatchedTrainWorkload, PlainTrainWorkload
    sc = synthetic.config_scene("c1")
    sc.targets = [np.random.default_rng(3).uniform(0, 1, (3, c.height, c.width)).astype(np.float32)
                  for c in sc.cameras]
    dev = torch.device("cuda")
    b = BatchedTrainWorkload(sc, dev, storage=torch.float32, tune=False)
    ms_b, lb = b.run(3)
    p = PlainTrainWorkload(sc, dev)
    ms_p, lp = p.run(3)
    assert lb[2] < lb[0]  # the replays advance: parameters and step count update
    for x, y in zip(lb, lp):
        assert abs(x - y) / y < 1e-4
    assert rel_err(b.geos.float(), p.geos.detach()) < 1e-4
    assert rel_err(b.shs.float(), p.shs.detach()) < 1e-4


def test_training_grid_step_graph_matches_plain_form():
    """Training grid points (the reference's parametrisation): the captured
    batched step (gather, render, backward, scatter, fused Adam over the grid
    and SH) tracks the plain per-view step with GatherGeoParams + SparseAdam."""
    from sv_raster_b200.workload import BatchedTrainWorkload, PlainTrainWorkload
    sc = synthetic.config_scene("c1")
    sc.targets = [np.random.default_rng(4).uniform(0, 1, (3, c.height, c.width)).astype(np.float32)
                  for c in sc.cameras]
    dev = torch.device("cuda")
    grid = synthetic.grid_params(sc, dev)
    b = BatchedTrainWorkload(sc, dev, storage=torch.float32, tune=False, grid=grid)
    _, lb = b.run(3)
    p = PlainTrainWorkload(sc, dev, grid=grid)
    _, lp = p.run(3)
    assert lb[2] < lb[0]
    for x, y in zip(lb, lp):
        assert abs(x - y) / y < 1e-4
    assert rel_err(b.grid.float(), p.grid.detach().reshape(-1)) < 1e-4


def _render_and_grads(r, C, wC, wT):
    r.fit_capacity(C.sh0, C.shs, 3)
    r.prepare(C.sh0, C.shs, 3)
    color, T = r.render(C.geos)
    dgeo, sub, dsh0, dshs = r.backward(C.geos, T, wC, wT, 3, 16)
    torch.cuda.synchronize()
    total, err = r.header()
    assert err == 0
    return color.clone(), T.clone(), dgeo.clone(), sub.clone(), dsh0.clone(), dshs.clone(), total


@pytest.mark.parametrize("tile,stage,order,ctas,buckets,lanes,binning,ppt", [
    (8, 64, (True, True), (0, 0), (512, 4096), 4, 1, 1),
    (8, 32, (True, False), (0, 0), (256, 4096), 1, 0, 1),
    (8, 128, (False, True), (0, 0), (1024, 2048), 2, 1, 1),
    (32, 256, (True, True), (0, 0), (512, 4096), 1, 0, 1),
    (16, 128, (True, True), (0, 0), (256, 2048), 8, 1, 1),
    (16, 512, (False, False), (0, 0), (1024, 4096), 2, 0, 1),
    (16, 256, (False, True), (3, 2), (512, 2048), 32, 0, 1),
    (8, 64, (True, True), (0, 0), (512, 4096), 1, 1, 2),
    (8, 32, (False, True), (0, 0), (512, 4096), 4, 1, 2),
    (16, 256, (True, False), (0, 0), (512, 4096), 1, 0, 2),
    (16, 128, (True, True), (0, 0), (512, 4096), 32, 1, 2),
])
def test_tiling_and_schedule_do_not_change_results(c1, tile, stage, order, ctas, buckets, lanes, binning, ppt):
    """Every tile size, staging depth, compositing schedule, sort-bucket
    setting and pixels per thread the autotuner may pick renders
    bit-identical images and T (a pixel
    sees the same instances in the same order) and the same gradients up to
    the order of the atomic additions."""
    g = torch.Generator(device="cuda").manual_seed(11)
    r0, _ = _raster(c1)
    n_pix = r0.n_pixels
    wC = torch.randn(3 * n_pix, device="cuda", generator=g)
    wT = torch.randn(n_pix, device="cuda", generator=g)
    base = _render_and_grads(r0, c1, wC, wT)
    r, _ = _raster(c1, tile_size=tile)
    r.set_staging(stage)
    r.set_schedule(fwd_ordered=order[0], bwd_ordered=order[1], fwd_ctas_per_sm=ctas[0], bwd_ctas_per_sm=ctas[1])
    r.set_sort_buckets(*buckets)
    r.set_reduction(lanes)
    r.set_binning(binning)
    r.set_pixels_per_thread(ppt)
    got = _render_and_grads(r, c1, wC, wT)
    assert torch.equal(got[0], base[0]), "colour differs"
    assert torch.equal(got[1], base[1]), "T differs"
    for a, b, name in zip(got[2:6], base[2:6], ("dL_dgeos", "subdiv", "dL_dsh0", "dL_dshs")):
        assert rel_err(a, b) < 1e-5, name
    if tile == 8:
        assert got[6] > base[6]  # smaller tiles duplicate more instances
    if tile == 32:
        assert got[6] < base[6]


@pytest.mark.parametrize("tile,stage,bstage", [(8, 64, 32), (8, 32, 128), (16, 256, 128)])
def test_backward_staging_depth_does_not_change_results(c1, tile, stage, bstage):
    """The backward's own staging depth (32 records: per-warp accumulators)
    gives the same gradients up to the order of additions."""
    g = torch.Generator(device="cuda").manual_seed(17)
    r0, _ = _raster(c1, tile_size=tile)
    r0.set_staging(stage)
    wC = torch.randn(3 * r0.n_pixels, device="cuda", generator=g)
    wT = torch.randn(r0.n_pixels, device="cuda", generator=g)
    base = _render_and_grads(r0, c1, wC, wT)
    r, _ = _raster(c1, tile_size=tile)
    r.set_staging(stage)
    r.set_backward_staging(bstage)
    got = _render_and_grads(r, c1, wC, wT)
    assert torch.equal(got[0], base[0])
    for a, b, name in zip(got[2:6], base[2:6], ("dL_dgeos", "subdiv", "dL_dsh0", "dL_dshs")):
        assert rel_err(a, b) < 1e-5, name


@pytest.mark.parametrize("ppt,bppt", [(1, 2), (2, 1)])
def test_backward_pixels_per_thread_apart(c1, ppt, bppt):
    """The backward's own pixels per thread: the same images and the same
    gradients up to the order of additions."""
    g = torch.Generator(device="cuda").manual_seed(23)
    r0, _ = _raster(c1, tile_size=8)
    r0.set_staging(32)
    wC = torch.randn(3 * r0.n_pixels, device="cuda", generator=g)
    wT = torch.randn(r0.n_pixels, device="cuda", generator=g)
    base = _render_and_grads(r0, c1, wC, wT)
    r, _ = _raster(c1, tile_size=8)
    r.set_staging(32)
    r.set_pixels_per_thread(ppt)
    r.set_backward_pixels_per_thread(bppt)
    got = _render_and_grads(r, c1, wC, wT)
    assert torch.equal(got[0], base[0]) and torch.equal(got[1], base[1])
    for a, b, name in zip(got[2:6], base[2:6], ("dL_dgeos", "subdiv", "dL_dsh0", "dL_dshs")):
        assert rel_err(a, b) < 1e-5, name


@pytest.mark.parametrize("views,grid_dtype,ppt", [((0, 1, 2), torch.float32, 2), ((0, 1, 2), torch.bfloat16, 1),
                                                  ("c3", torch.float32, 2)])
def test_grid_fused_matches_separate(c1, views, grid_dtype, ppt):
    """Grid-point densities read while staging and corner gradients added
    into the grid in the flush (svr_batch_render_grid / _backward_grid)
    against the separate all-voxel gather and scatter around render /
    backward: images and T bitwise, grid gradient to the order of additions,
    also through the autograd function (fused=True vs False)."""
    if views == "c3":
        C = SceneTensors(synthetic.cached_config_scene("c3"))
        cams = [DevCam(C.scene.cameras[i]) for i in (0, 5)]
    else:
        C = c1
        cams = [DevCam(C.scene.cameras[i]) for i in views]
    from sv_raster_b200.batched import GridBatchedRender, gather_grid_geos, scatter_grid_grad
    key, grid_np = synthetic.grid_params(C.scene, torch.device("cuda"))
    key = key.contiguous()
    grid = torch.from_numpy(grid_np).cuda().to(grid_dtype)
    M = grid.numel()
    r = BatchedRasterizer(cams, C.octpath, C.centers, C.lengths, max_level=C.scene.max_level, tile_size=8)
    r.set_backward_pixels_per_thread(ppt)
    r.fit_capacity(C.sh0, C.shs, 3)
    r.prepare(C.sh0, C.shs, 3)
    g = torch.Generator(device="cuda").manual_seed(31)
    wC = torch.randn(3 * r.n_pixels, device="cuda", generator=g)
    wT = torch.randn(r.n_pixels, device="cuda", generator=g)
    P = C.centers.shape[0]
    geos = torch.empty(P, 8, dtype=grid_dtype, device="cuda")
    gather_grid_geos(key, grid, geos)
    color_a, T_a = r.render(geos)
    dgeo = torch.zeros(P, 8, device="cuda")
    r.backward_render(geos, T_a, wC, wT, dgeo)
    dgrid_a = torch.zeros(M, device="cuda")
    scatter_grid_grad(key, dgeo, dgrid_a)
    color_b, T_b = r.render_grid(key, grid)
    dgrid_b = torch.zeros(M, device="cuda")
    r.backward_render_grid(key, grid, T_b, wC, wT, dgrid_b)
    torch.cuda.synchronize()
    assert r.header()[1] == 0
    assert torch.equal(color_a, color_b) and torch.equal(T_a, T_b)
    err = rel_err(dgrid_b, dgrid_a)
    print(f"fused grid ({views}, {grid_dtype}, {ppt} px/thread bwd): grid gradient rel {err:.2e}")
    assert err < 1e-5
    grads = {}
    for fused in (False, True):
        gp = grid.clone().requires_grad_(True)
        s0 = C.sh0.clone().requires_grad_(True)
        s1 = C.shs.clone().requires_grad_(True)
        col, T = GridBatchedRender.apply(r, 3, key, gp, s0, s1, fused)
        ((col * wC).sum() + (T * wT).sum()).backward()
        grads[fused] = (col.detach(), gp.grad.float(), s0.grad, s1.grad)
    assert torch.equal(grads[True][0], grads[False][0])
    tol = 1e-5 if grid_dtype == torch.float32 else 1e-2  # bf16 gradients round differently per summation order
    for a_, b_ in zip(grads[True][1:], grads[False][1:]):
        assert rel_err(a_, b_) < tol


def test_autotuner_runs_and_keeps_results(c1, tmp_path, monkeypatch):
    from sv_raster_b200.autotune import tune_batched
    monkeypatch.setenv("SVR_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    g = torch.Generator(device="cuda").manual_seed(5)
    r0, _ = _raster(c1)
    wC = torch.randn(3 * r0.n_pixels, device="cuda", generator=g)
    wT = torch.randn(r0.n_pixels, device="cuda", generator=g)
    base = _render_and_grads(r0, c1, wC, wT)
    r, _ = _raster(c1)
    res = tune_batched(r, c1.geos, c1.sh0, c1.shs, 3, reps=2, warmup=1)
    assert not res["cached"] and set(res["choice"]) == {"tile", "ppt", "bppt", "bstage", "fstage", "bin", "sort",
                                                        "fwd", "bwd", "reduce"}
    got = _render_and_grads(r, c1, wC, wT)
    assert torch.equal(got[0], base[0])
    assert rel_err(got[2], base[2]) < 1e-5
    r2, _ = _raster(c1)
    res2 = tune_batched(r2, c1.geos, c1.sh0, c1.shs, 3)
    assert res2["cached"] and res2["choice"] == res["choice"]
    assert r2.tile_size == res["choice"]["tile"][0]
