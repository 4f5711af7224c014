"""Setup utilities and the svraster_cuda drop-in shim (CPU)."""
import numpy as np
import torch

from sv_raster_b200 import synthetic, utils


def test_octpath_utils_match_generator():
    sc = synthetic.config_scene("c1", n_voxels=3000)
    lv = torch.from_numpy(sc.octlevel)
    ijk = torch.from_numpy(synthetic.octpath_to_ijk(sc.octpath, sc.octlevel))
    path = utils.ijk_2_octpath(ijk, lv)
    assert torch.equal(path.reshape(-1), torch.from_numpy(sc.octpath))
    assert torch.equal(utils.octpath_2_ijk(path, lv), ijk)


def test_voxel_order_rank():
    p = torch.tensor([0, 5 << 45, 123456789], dtype=torch.int64)
    r = utils.voxel_order_rank(p)
    assert r.shape == (8, 3)
    rep = sum(7 << (3 * l) for l in range(16))
    assert int(r[7, 0]) == rep and int(r[0, 1]) == 5 << 45
    assert torch.equal(r[3] ^ r[0], torch.full((3,), sum(3 << (3 * l) for l in range(16)), dtype=torch.int64))


def test_compute_rd_and_depth2pts():
    cam = synthetic.make_camera(8, 6, 60.0, (0.1, 0.2, -1.0))
    c2w = torch.from_numpy(cam.c2w)
    rd = utils.compute_rd(8, 6, cam.cx, cam.cy, cam.tanfovx, cam.tanfovy, c2w)
    assert rd.shape == (3, 6, 8)
    # centre-ish pixel looks towards the target (the origin)
    d = rd[:, 3, 4] / rd[:, 3, 4].norm()
    fwd = -torch.from_numpy(cam.c2w[:3, 3]) / np.linalg.norm(cam.c2w[:3, 3])
    assert float(d @ fwd) > 0.99
    depth = torch.full((6, 8), 2.0)
    pts = utils.depth2pts(8, 6, cam.cx, cam.cy, cam.tanfovx, cam.tanfovy, c2w, depth)
    assert torch.allclose(pts, torch.from_numpy(cam.c2w[:3, 3])[:, None, None] + 2.0 * rd)


def test_is_in_cone():
    cam = synthetic.make_camera(64, 48, 60.0, (0.0, 0.0, -1.0))

    class C:
        w2c = torch.from_numpy(cam.w2c)
        tanfovx, tanfovy, near = cam.tanfovx, cam.tanfovy, 0.02
    pts = torch.tensor([[0.0, 0.0, 0.0], [0.0, 0.0, -2.0], [5.0, 0.0, 0.0]])
    assert utils.is_in_cone(pts, C).tolist() == [True, False, False]


def test_svraster_cuda_shim_resolves_to_this_package():
    import sv_raster_b200
    mod = sv_raster_b200.install_as_svraster_cuda()
    import svraster_cuda.renderer
    import svraster_cuda.sparse_adam
    from svraster_cuda.meta import MAX_NUM_LEVELS, STEP_SZ_SCALE
    assert mod.renderer is sv_raster_b200.renderer
    assert svraster_cuda.sparse_adam.SparseAdam is sv_raster_b200.sparse_adam.SparseAdam
    assert MAX_NUM_LEVELS == 16 and STEP_SZ_SCALE == 100.0
    assert hasattr(svraster_cuda.grid_loss_bw, "total_variation")


def test_levels21_surface_imports_with_its_depth():
    """The new_svraster_cuda drop-in: the same modules over a 21-level _C."""
    import importlib
    import sys
    from sv_raster_b200 import levels21
    assert levels21._C.MAX_NUM_LEVELS == 21 and levels21.meta.MAX_NUM_LEVELS == 21
    assert levels21.utils.MAX_NUM_LEVELS == 21 and levels21.meta.MAX_SORT_KEY_BITS == 128
    assert levels21.meta.MAX_RENDER_TILES == 4096 * 4096
    assert levels21.renderer._C is levels21._C
    from sv_raster_b200 import renderer, utils
    assert renderer._C.MAX_NUM_LEVELS == 16 and utils.MAX_NUM_LEVELS == 16
    compat = __import__("os").path.join(__import__("os").path.dirname(renderer.__file__), "compat")
    sys.path.insert(0, compat)
    try:
        m = importlib.import_module("new_svraster_cuda")
        assert m.renderer is levels21.renderer and m.meta.MAX_NUM_LEVELS == 21
    finally:
        sys.path.remove(compat)


def test_deep_scene_spans_21_levels():
    from sv_raster_b200 import synthetic
    sc = synthetic.deep_scene(n_voxels=3000, n_chains=8)
    assert int(sc.octlevel.min()) == 6 and int(sc.octlevel.max()) == 21
    assert int(sc.octpath.max()).bit_length() > 48  # ranks use the bits below a 16-level path
    c, l = synthetic.decode_voxels(sc.octpath, sc.octlevel, 21)
    assert (c == sc.centers).all() and (l == sc.lengths).all()
