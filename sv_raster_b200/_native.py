"""ctypes binding of ``libsvr_b200.so`` (the C ABI declared in include/svr_b200.h).

The library is loaded from the package directory.  There is no fallback: if
the library is missing or fails to load, every hot-path op raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsvr_b200.so")

c_int = ctypes.c_int
c_i64 = ctypes.c_int64
c_f = ctypes.c_float
c_d = ctypes.c_double
c_sz = ctypes.c_size_t
c_p = ctypes.c_void_p


class Camera(ctypes.Structure):
    """Mirror of ``svr_camera``."""
    _fields_ = [
        ("width", c_int), ("height", c_int),
        ("tanfovx", c_f), ("tanfovy", c_f),
        ("cx", c_f), ("cy", c_f),
        ("w2c", c_p), ("c2w", c_p),
        ("near_plane", c_f), ("bg_color", c_f),
    ]


# name -> (restype, argtypes)
_SIGS = {
    "svr_max_num_levels": (c_int, []),
    "svr_step_sz_scale": (c_f, []),
    "svr_max_n_samp": (c_int, []),
    "svr_status_string": (ctypes.c_char_p, [c_int]),
    "svr_version": (c_int, []),
    "svr_geom_buffer_bytes": (c_sz, [c_i64]),
    "svr_image_buffer_bytes": (c_sz, [c_int, c_int]),
    "svr_binning_buffer_bytes": (c_sz, [c_i64, c_int, c_int]),
    "svr_rasterize_preprocess": (c_int, [ctypes.POINTER(Camera), c_i64, c_p, c_p, c_p, c_p, c_p, c_sz, c_int, c_p]),
    "svr_rasterize_preprocess_noalloc": (c_int, [ctypes.POINTER(Camera), c_i64, c_p, c_p, c_p, c_p, c_p, c_sz, c_int,
                                                 c_p]),
    "svr_noalloc_max_voxels": (c_i64, []),
    "svr_geom_count_ptr": (c_p, [c_p]),
    "svr_geom_error_ptr": (c_p, [c_p]),
    "svr_rasterize_forward": (c_int, [ctypes.POINTER(Camera), c_int, c_int, c_int, c_int, c_int, c_i64, c_i64,
                                      c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_sz, c_p, c_sz,
                                      c_p, c_p, c_p, c_p, c_p, c_int, c_p]),
    "svr_rasterize_binning": (c_int, [ctypes.POINTER(Camera), c_i64, c_i64, c_p, c_p, c_p, c_sz, c_p, c_sz, c_int,
                                      c_p]),
    "svr_rasterize_render": (c_int, [ctypes.POINTER(Camera), c_int, c_int, c_int, c_int, c_int, c_i64, c_i64,
                                     c_p, c_p, c_p, c_p, c_p, c_p, c_sz, c_p, c_sz, c_p, c_p, c_p, c_p, c_p, c_int,
                                     c_p]),
    "svr_rasterize_backward": (c_int, [ctypes.POINTER(Camera), c_int, c_i64, c_i64,
                                       c_p, c_p, c_p, c_p, c_p, c_p, c_p,
                                       c_p, c_p, c_p, c_p, c_p, c_f, c_p, c_f, c_f, c_int, c_int,
                                       c_p, c_p, c_p, c_p, c_p, c_int, c_p]),
    "svr_unpack_image_state": (c_int, [c_int, c_int, c_p, c_p, c_p, c_p, c_p]),
    "svr_binning_sorted": (c_int, [c_p, c_i64, c_int, c_int, ctypes.POINTER(c_p), ctypes.POINTER(c_p)]),
    "svr_binning_sorted_wide": (c_int, [c_p, c_i64, c_int, c_int, ctypes.POINTER(c_p), ctypes.POINTER(c_p),
                                        ctypes.POINTER(c_p)]),
    "svr_binning_buffer_bytes_levels": (c_sz, [c_i64, c_int, c_int, c_int]),
    "svr_rasterize_binning_levels": (c_int, [ctypes.POINTER(Camera), c_i64, c_i64, c_p, c_int, c_p, c_p, c_sz, c_p,
                                             c_sz, c_int, c_p]),
    "svr_rasterize_forward_levels": (c_int, [ctypes.POINTER(Camera), c_int, c_int, c_int, c_int, c_int, c_i64, c_i64,
                                             c_p, c_int, c_p, c_p, c_p, c_p, c_p, c_p, c_sz, c_p, c_sz,
                                             c_p, c_p, c_p, c_p, c_p, c_int, c_p]),
    "svr_geom_arrays": (c_int, [c_p, c_i64, ctypes.POINTER(c_p), ctypes.POINTER(c_p), ctypes.POINTER(c_p),
                                ctypes.POINTER(c_p)]),
    "svr_sh_compute": (c_int, [c_int, c_i64, c_p, c_i64, c_int, c_p, c_p, c_p, c_p, c_int, c_p, c_p]),
    "svr_sh_compute_bw": (c_int, [c_int, c_int, c_i64, c_p, c_i64, c_p, c_p, c_p, c_p, c_p, c_p]),
    "svr_unbiased_adam_step": (c_int, [c_int, c_i64, c_p, c_p, c_p, c_p, c_d, c_d, c_d, c_d, c_f, c_p]),
    "svr_biased_adam_step": (c_int, [c_int, c_i64, c_p, c_p, c_p, c_p, c_f, c_f, c_f, c_f, c_p]),
    "svr_fused_adam_step": (c_int, [c_int, c_int, ctypes.POINTER(c_p), ctypes.POINTER(c_int), ctypes.POINTER(c_p),
                                    ctypes.POINTER(c_p), ctypes.POINTER(c_p), ctypes.POINTER(c_i64),
                                    ctypes.POINTER(c_d), ctypes.POINTER(c_d), c_d, c_d, c_f, c_p]),
    "svr_fused_adam_step_device": (c_int, [c_int, c_int, ctypes.POINTER(c_p), ctypes.POINTER(c_int),
                                           ctypes.POINTER(c_p), ctypes.POINTER(c_p), ctypes.POINTER(c_p),
                                           ctypes.POINTER(c_i64), ctypes.POINTER(c_d), c_d, c_d, c_f, c_p, c_p]),
    "svr_gather_grid_params": (c_int, [c_int, c_i64, c_p, c_p, c_p, c_p, c_p]),
    "svr_gather_grid_params_bw": (c_int, [c_int, c_i64, c_p, c_p, c_p, c_p, c_p]),
    "svr_gather_grid_geo_all": (c_int, [c_i64, c_p, c_p, c_int, c_p, c_int, c_p]),
    "svr_scatter_grid_geo_all": (c_int, [c_i64, c_p, c_p, c_p, c_p]),
    "svr_read_error": (c_int, [c_p, ctypes.POINTER(ctypes.c_uint32), c_p]),
    "svr_total_variation_bw": (c_int, [c_p, c_p, c_f, c_p, c_int, c_int, c_i64, c_int, c_p, c_p, c_p]),
    "svr_batch_plan_create": (c_int, [c_int, ctypes.POINTER(Camera), c_i64, c_i64, c_int, c_int, c_int,
                                      ctypes.POINTER(c_p), ctypes.POINTER(c_sz)]),
    "svr_batch_plan_destroy": (None, [c_p]),
    "svr_batch_plan_set_schedule": (c_int, [c_p, c_int, c_int, c_int]),
    "svr_batch_plan_invalidate_geometry": (c_int, [c_p]),
    "svr_batch_plan_set_sort_buckets": (c_int, [c_p, c_int, c_int]),
    "svr_batch_plan_set_staging": (c_int, [c_p, c_int]),
    "svr_batch_plan_tile_size": (c_int, [c_p]),
    "svr_batch_plan_set_reduction": (c_int, [c_p, c_int]),
    "svr_batch_plan_set_arithmetic": (c_int, [c_p, c_int]),
    "svr_batch_plan_set_culling": (c_int, [c_p, c_int]),
    "svr_batch_plan_set_backward_staging": (c_int, [c_p, c_int]),
    "svr_batch_plan_set_pixels_per_thread": (c_int, [c_p, c_int]),
    "svr_batch_plan_set_backward_pixels_per_thread": (c_int, [c_p, c_int]),
    "svr_batch_plan_set_binning": (c_int, [c_p, c_int]),
    "svr_batch_plan_pixels": (c_i64, [c_p]),
    "svr_batch_plan_tiles": (c_i64, [c_p]),
    "svr_batch_plan_groups": (c_int, [c_p]),
    "svr_batch_count_ptr": (c_p, [c_p, c_p]),
    "svr_batch_error_ptr": (c_p, [c_p, c_p]),
    "svr_batch_bbox_ptr": (c_p, [c_p, c_p]),
    "svr_batch_arrays": (c_int, [c_p, c_p] + [ctypes.POINTER(c_p)] * 7),
    "svr_batch_prepare": (c_int, [c_p, c_p, c_p, c_p, c_p, c_p, c_p, c_int, c_int, c_int, c_p]),
    "svr_batch_render": (c_int, [c_p, c_p, c_p, c_p, c_p, c_int, c_p, c_p, c_p]),
    "svr_batch_backward": (c_int, [c_p, c_p, c_p, c_p, c_p, c_int, c_p, c_p, c_p, c_p, c_p]),
    "svr_batch_render_grid": (c_int, [c_p, c_p, c_p, c_p, c_p, c_p, c_int, c_p, c_p, c_p]),
    "svr_batch_backward_grid": (c_int, [c_p, c_p, c_p, c_p, c_p, c_p, c_int, c_p, c_p, c_p, c_p, c_p]),
    "svr_batch_sh_backward": (c_int, [c_p, c_p, c_p, c_int, c_int, c_p, c_p, c_p, c_p]),
}

_lib = None
_load_error = None


def lib():
    """The loaded library (raises ``RuntimeError`` if it cannot be loaded)."""
    global _lib, _load_error
    if _lib is not None:
        return _lib
    if _load_error is not None:
        raise RuntimeError(_load_error)
    if not os.path.exists(LIB_PATH):
        _load_error = (f"sv_raster_b200: native library not built ({LIB_PATH}); "
                       "run `python -m sv_raster_b200.build`")
        raise RuntimeError(_load_error)
    try:
        L = ctypes.CDLL(LIB_PATH)
    except OSError as e:  # pragma: no cover - depends on the host
        _load_error = f"sv_raster_b200: failed to load {LIB_PATH}: {e}"
        raise RuntimeError(_load_error) from e
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols():
    return sorted(_SIGS)


def check(status, what):
    if status != 0:
        msg = lib().svr_status_string(status).decode()
        raise RuntimeError(f"{what} failed: {msg} (status {status})")
