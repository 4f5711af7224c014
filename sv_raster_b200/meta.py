"""Compile-time constants (reference backends/cuda/svraster_cuda/meta.py, config.h:16-23; the 21-level
surface adds new_cuda's sort-key and packed-bbox limits, new_svraster_cuda/meta.py:15-17)."""
from . import _C

MAX_NUM_LEVELS = _C.MAX_NUM_LEVELS
STEP_SZ_SCALE = _C.STEP_SZ_SCALE
MAX_N_SAMP = _C.MAX_N_SAMP

for _name in ("MAX_SORT_KEY_BITS", "MAX_PACKED_IMAGE_DIM", "MAX_RENDER_TILES"):
    if hasattr(_C, _name):
        globals()[_name] = getattr(_C, _name)
