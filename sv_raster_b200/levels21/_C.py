"""Native ops for octrees 21 levels deep, with the surface of the reference's
``new_svraster_cuda._C`` (backends/new_cuda/binding.cpp): the ops of
``sv_raster_b200._C`` with the forward bound to 21-level binning (63-bit
Morton ranks, (tile, rank) keys wider than 64 bits; new_cuda
forward.cu:660-752) and the new backend's three extra constants
(config.h:24-34, binding.cpp:55-57).  Every other op is unchanged by the
octree depth."""
from .. import _C as _base
from .._C import *  # noqa: F401,F403  (the ops that do not depend on the depth)

MAX_NUM_LEVELS = 21
STEP_SZ_SCALE = _base.STEP_SZ_SCALE
MAX_N_SAMP = _base.MAX_N_SAMP
MAX_SORT_KEY_BITS = 128
MAX_PACKED_IMAGE_DIM = (1 << 16) - 1
MAX_RENDER_TILES = ((MAX_PACKED_IMAGE_DIM + 16) // 16) ** 2


def rasterize_voxels(n_samp_per_vox, image_width, image_height, tan_fovx, tan_fovy, cx, cy, w2c_matrix, c2w_matrix,
                     bg_color, need_depth, need_distortion, need_normal, track_max_w, octree_paths, vox_centers,
                     vox_lengths, geos, rgbs, geomBuffer, debug=False):
    """new_cuda forward.cu:783-870 -> (num_rendered, binningBuffer, imgBuffer, color, depth, normal, T, max_w)."""
    return _base.rasterize_voxels(n_samp_per_vox, image_width, image_height, tan_fovx, tan_fovy, cx, cy, w2c_matrix,
                                  c2w_matrix, bg_color, need_depth, need_distortion, need_normal, track_max_w,
                                  octree_paths, vox_centers, vox_lengths, geos, rgbs, geomBuffer, debug,
                                  levels=MAX_NUM_LEVELS)


def unpack_sorted_list(binningBuffer, num_rendered, width, height):
    """(keys_hi, keys_lo, values) of a 21-level binning buffer: the sorted
    128-bit keys as the reference's SortKey128 halves, and the sorted values."""
    return _base.unpack_sorted_list_wide(binningBuffer, num_rendered, width, height)
