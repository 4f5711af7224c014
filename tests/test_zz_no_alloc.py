"""The scratch-free projection entry point, through the C ABI.

svr_rasterize_preprocess_noalloc serves callers that cannot allocate device
memory (an embedding application that owns every device buffer, capture-time
code, real-time loops): its scan scratch is a static device array of the
library.  It must produce exactly what svr_rasterize_preprocess produces
(integers: duplicate counts, scan, packed bboxes, quadrant bitsets, instance
count), call after call, although every call reuses the same array.  This
file is collected last so a failure here does not hide the others.
"""
import ctypes

import numpy as np
import pytest
import torch

from sv_raster_b200 import _native, synthetic

pytestmark = pytest.mark.gpu


def _camera(cam, w2c, c2w):
    return _native.Camera(cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, w2c.data_ptr(),
                          c2w.data_ptr(), cam.near, 0.0)


def _run(fn, cam, w2c, c2w, octpath, centers, lengths):
    L = _native.lib()
    P = centers.shape[0]
    nbytes = L.svr_geom_buffer_bytes(P)
    geom = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    ndup = torch.zeros(P, dtype=torch.int32, device="cuda")
    c = _camera(cam, w2c, c2w)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    st = fn(ctypes.byref(c), P, p(octpath), p(centers), p(lengths), p(ndup), p(geom), nbytes, 0, stream)
    assert st == 0, L.svr_status_string(st)
    torch.cuda.synchronize()
    arrays = [ctypes.c_void_p() for _ in range(4)]
    assert L.svr_geom_arrays(p(geom), P, *[ctypes.byref(a) for a in arrays]) == 0
    base = geom.data_ptr()
    off = [a.value - base for a in arrays]
    out = dict(ndup=ndup.cpu().numpy(), count=int(geom[:4].view(torch.int32).item()) & 0xFFFFFFFF,
               err=int(geom[4:8].view(torch.int32).item()),
               scan=geom[off[1]:off[1] + 4 * P].view(torch.int32).cpu().numpy(),
               bbox=geom[off[2]:off[2] + 8 * P].view(torch.int32).cpu().numpy().reshape(P, 2),
               quad=geom[off[3]:off[3] + 4 * P].view(torch.int32).cpu().numpy())
    return out


def _tensors(sc):
    t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)
    return t(sc.octpath.reshape(-1, 1), torch.int64), t(sc.centers), t(sc.lengths)


@pytest.mark.parametrize("n_voxels", [20000, 300000])
def test_noalloc_preprocess_matches_the_allocating_entry_point(n_voxels):
    L = _native.lib()
    sc = synthetic.config_scene("c1", n_voxels=n_voxels)
    octpath, centers, lengths = _tensors(sc)
    # two calls in a row, different cameras: the shared scratch keeps the
    # previous call's partial sums and must not leak into the next result
    for cam in (sc.cameras[0], sc.cameras[2], sc.cameras[1]):
        w2c = torch.from_numpy(cam.w2c).cuda()
        c2w = torch.from_numpy(cam.c2w).cuda()
        want = _run(L.svr_rasterize_preprocess, cam, w2c, c2w, octpath, centers, lengths)
        got = _run(L.svr_rasterize_preprocess_noalloc, cam, w2c, c2w, octpath, centers, lengths)
        assert got["err"] == 0 and want["err"] == 0
        assert got["count"] == want["count"] > 0
        assert np.array_equal(got["ndup"], want["ndup"])
        assert np.array_equal(got["scan"], want["scan"])
        vis = want["ndup"] > 0
        assert np.array_equal(got["bbox"][vis], want["bbox"][vis])
        assert np.array_equal(got["quad"][vis], want["quad"][vis])
        assert got["count"] == int(want["ndup"].astype(np.int64).sum())


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = _native.lib()
    limit = L.svr_noalloc_max_voxels()
    assert limit == 4096 * 16384
    dummy = torch.zeros(16, device="cuda")
    cam = _native.Camera(64, 48, 0.5, 0.4, 32.0, 24.0, dummy.data_ptr(), dummy.data_ptr(), 0.02, 0.0)
    st = L.svr_rasterize_preprocess_noalloc(ctypes.byref(cam), limit + 1, None, ctypes.c_void_p(dummy.data_ptr()),
                                            ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(dummy.data_ptr()),
                                            ctypes.c_void_p(dummy.data_ptr()), 0, 0, None)
    assert st == 2  # SVR_ERR_CAPACITY, nothing launched
    assert L.svr_status_string(st) == b"buffer capacity exceeded"
