"""Compile-time constants (reference backends/cuda/svraster_cuda/meta.py, config.h:16-23)."""
from . import _C

MAX_NUM_LEVELS = _C.MAX_NUM_LEVELS
STEP_SZ_SCALE = _C.STEP_SZ_SCALE
MAX_N_SAMP = _C.MAX_N_SAMP
