"""Parity with the reference's new_cuda backend: octrees 21 levels deep.

The reference's new_cuda backend (compiled from its own sources into
oracle/_ref/new_svraster_ref_C.so) and this repository's 21-level surface
(``sv_raster_b200.levels21``, the ``new_svraster_cuda`` drop-in) run on the
same seeded scene: the c1 sphere with chains of voxels refined down to level
21, so the 63-bit Morton ranks differ below the 48 bits of a 16-level octree.
Views of 1 and 2 tiles keep the reference on its 64-bit keys
(forward.cu:666-685 of new_cuda); larger views use its 128-bit keys.

Bit-exact: duplicate counts, bboxes, quadrants, the instance count, the
sorted keys (both halves of the wide keys) and values, tile ranges,
tile_last and contributor counts.  Bitwise: images and T.  Gradients within
1e-5 norm-wise.
"""
import pytest
import torch

from refutil import SceneTensors, align128, ref_binning_sorted, ref_geom_arrays, rel_err, run_bwd, run_view
from sv_raster_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref21():
    import build_ref
    try:
        return build_ref.load("new_cuda")
    except ImportError as e:
        pytest.skip(f"new_cuda reference checker not built: {e}")


@pytest.fixture(scope="module")
def deep():
    sc = synthetic.deep_scene()
    sc.cameras = sc.cameras + [synthetic.make_camera(16, 16, 20.0, (0.0, 0.0, -1.5)),
                               synthetic.make_camera(32, 16, 30.0, (0.4, 0.2, -1.3)),
                               synthetic.make_camera(1920, 1080, 50.0, (0.9, -0.4, -1.2))]
    return SceneTensors(sc)


def ref_binning_sorted_wide(binning, R):
    """Sorted SortKey128 {hi, lo} keys and values of a new_cuda wide-key
    binning buffer (raster_state.cu:101-140 of new_cuda: wide unsorted keys,
    wide keys, unsorted values, values, each 128-byte aligned)."""
    o_ku = 0
    o_k = align128(o_ku + 16 * R)
    o_vu = align128(o_k + 16 * R)
    o_v = align128(o_vu + 4 * R)
    keys = binning[o_k:o_k + 16 * R].view(torch.int64).view(R, 2)
    return keys[:, 0], keys[:, 1], binning[o_v:o_v + 4 * R].view(torch.int32)


@pytest.mark.parametrize("cam_i", [0, 1, 2, 3, 4, 5])
def test_levels21_matches_new_cuda_reference(ref21, deep, cam_i):
    from sv_raster_b200.levels21 import _C as C21
    assert C21.MAX_NUM_LEVELS == ref21.MAX_NUM_LEVELS == 21
    assert (C21.MAX_SORT_KEY_BITS, C21.MAX_PACKED_IMAGE_DIM, C21.MAX_RENDER_TILES) == \
        (ref21.MAX_SORT_KEY_BITS, ref21.MAX_PACKED_IMAGE_DIM, ref21.MAX_RENDER_TILES)
    C = deep
    P = C.centers.shape[0]
    a = run_view(C21, C, cam_i, 1)
    b = run_view(ref21, C, cam_i, 1, rgbs=a["rgbs"])
    torch.cuda.synchronize()
    assert torch.equal(a["ndup"], b["ndup"])
    nd, _, bb, qd = C21.unpack_geom_state(a["geom"], P)[:4]
    rnd, rbb, rqd = ref_geom_arrays(b["geom"], P)
    vis = rnd > 0
    assert torch.equal(bb[vis], rbb[vis]) and torch.equal(qd[vis], rqd[vis])
    assert a["R"] == b["R"] and a["R"] > 0
    R, cam = a["R"], a["cam"]
    hi, lo, v = C21.unpack_sorted_list(a["binning"], R, cam.width, cam.height)
    n_tiles = ((cam.width + 15) // 16) * ((cam.height + 15) // 16)
    if n_tiles <= 2:  # the reference's 64-bit keys: tile << 63 | rank
        rk, rv = ref_binning_sorted(b["binning"], R)
        assert torch.equal(lo, rk), "sorted keys differ"
        assert not bool(hi.any())
    else:
        rhi, rlo, rv = ref_binning_sorted_wide(b["binning"], R)
        assert torch.equal(lo, rlo) and torch.equal(hi, rhi), "sorted wide keys differ"
    assert torch.equal(v, rv), "sorted values differ"
    ra, ta, na = C21.unpack_ImageState(cam.width, cam.height, a["img"])
    rr, rt, rn = ref21.unpack_ImageState(cam.width, cam.height, b["img"])
    assert torch.equal(ra, rr) and torch.equal(ta, rt) and torch.equal(na, rn)
    assert torch.equal(a["color"], b["color"]) and torch.equal(a["T"], b["T"])
    g = torch.Generator(device="cuda").manual_seed(cam_i)
    dC = torch.randn(a["color"].shape, device="cuda", generator=g) * 1e-3
    dT = torch.randn(a["T"].shape, device="cuda", generator=g) * 1e-3
    ga = run_bwd(C21, C, a, 1, dC, dT)
    gb = run_bwd(ref21, C, b, 1, dC, dT)
    for x, y, name in zip(ga, gb, ("dL_dgeos", "dL_drgbs", "subdiv_p_bw")):
        assert rel_err(x, y) <= 1e-5, name
    if cam_i in (0, 1, 5):  # views of the whole sphere: the deepest voxels are in the lists
        levels = C.octlevel.reshape(-1).long()
        assert int(levels[v.long() & ((1 << 29) - 1)].max()) == 21
