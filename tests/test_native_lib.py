"""The C-ABI library: it loads, exports exactly what include/svr_b200.h
declares, and the host-side checks of the Python surface behave like the
reference's (no GPU needed)."""
import ctypes
import os
import re

import pytest
import torch

from conftest import ROOT
from sv_raster_b200 import _native, renderer
from sv_raster_b200.build import LIB, build


def header_functions():
    src = open(os.path.join(ROOT, "include", "svr_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(svr_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    build()
    return _native.lib()


def test_library_builds_and_loads(lib):
    assert os.path.exists(LIB)
    assert lib.svr_version() >= 1


def test_exports_match_header(lib):
    declared = header_functions()
    assert declared, "no declarations parsed"
    raw = ctypes.CDLL(LIB)
    for name in declared:
        assert hasattr(raw, name), f"{name} declared but not exported"
    assert sorted(_native.exported_symbols()) == declared


def test_constants(lib):
    assert lib.svr_max_num_levels() == 16
    assert lib.svr_step_sz_scale() == 100.0
    assert lib.svr_max_n_samp() == 3
    assert lib.svr_status_string(2) == b"buffer capacity exceeded"


def test_buffer_sizes(lib):
    g1, g2 = lib.svr_geom_buffer_bytes(1000), lib.svr_geom_buffer_bytes(2000)
    assert 0 < g1 < g2 and g1 >= 1000 * 20
    assert lib.svr_image_buffer_bytes(256, 256) >= 256 * 256 * 4 + 256 * 12
    assert lib.svr_binning_buffer_bytes(10000, 256, 256) >= 10000 * 24
    assert lib.svr_geom_buffer_bytes(-1) == 0


def test_invalid_arguments_rejected_without_device(lib):
    cam = _native.Camera(0, 0, 0.5, 0.5, 0.0, 0.0, None, None, 0.02, 0.0)
    st = lib.svr_rasterize_preprocess(ctypes.byref(cam), 10, None, None, None, None, None, 0, 0, None)
    assert st == 1  # SVR_ERR_SHAPE
    st = lib.svr_sh_compute(4, 0, None, 10, 16, None, None, None, None, 0, None, None)
    assert st == 1
    st = lib.svr_fused_adam_step(9, 0, None, None, None, None, None, None, None, None, 0.9, 0.99, 1e-15, None)
    assert st == 1


def _settings(**kw):
    eye = torch.eye(4)
    base = dict(color_mode="sh", n_samp_per_vox=1, image_width=16, image_height=16, tanfovx=0.5, tanfovy=0.5,
                cx=8.0, cy=8.0, w2c_matrix=eye, c2w_matrix=eye)
    base.update(kw)
    return renderer.RasterSettings(**base)


def test_python_surface_checks_like_reference():
    paths = torch.zeros(4, 1, dtype=torch.int64)
    cen = torch.zeros(4, 3)
    ln = torch.ones(4, 1)
    with pytest.raises(Exception, match="Expect RasterSettings"):
        renderer.rasterize_voxels(None, paths, cen, ln, None)
    with pytest.raises(Exception, match="n_samp_per_vox"):
        renderer.rasterize_voxels(_settings(n_samp_per_vox=4), paths, cen, ln, None)
    with pytest.raises(Exception, match="Size mismatched"):
        renderer.rasterize_voxels(_settings(), paths, cen[:3], ln, None)
    with pytest.raises(Exception, match=r"shape \[N, 3\]"):
        renderer.rasterize_voxels(_settings(), paths, torch.zeros(4, 2), ln, None)
    with pytest.raises(ValueError):
        from sv_raster_b200.sparse_adam import SparseAdam
        SparseAdam([torch.zeros(3, requires_grad=True)], lr=-1.0)
