"""The operator surface of the reference's ``new_svraster_cuda`` package
(backends/new_cuda): octrees 21 levels deep.

The reference's new package keeps the Python modules of the 16-level one
(renderer, sparse_adam, utils, grid_loss_bw; only meta adds constants).  Here
the modules that reach the octree depth through ``_C`` (renderer, utils,
meta) are those of ``sv_raster_b200`` executed again with this package's
``_C`` (21-level forward, ``MAX_NUM_LEVELS = 21``); sparse_adam and
grid_loss_bw do not depend on the depth and are shared.
"""
import importlib.util
import os
import sys

from .. import grid_loss_bw, sparse_adam  # noqa: F401  (independent of the octree depth)
from . import _C  # noqa: F401

_BASE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load(name):
    full = f"{__name__}.{name}"
    if full in sys.modules:
        return sys.modules[full]
    spec = importlib.util.spec_from_file_location(full, os.path.join(_BASE, f"{name}.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[full] = mod
    spec.loader.exec_module(mod)
    return mod


meta = _load("meta")
utils = _load("utils")
renderer = _load("renderer")

__all__ = ["_C", "meta", "utils", "renderer", "sparse_adam", "grid_loss_bw"]
