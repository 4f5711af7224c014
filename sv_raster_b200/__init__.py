"""sm_100a sparse-voxel rasterizer with the operator surface of SVRaster's
``svraster_cuda`` backend (renderer, sparse_adam, meta, utils, grid_loss_bw),
plus a multi-view batched path (``sv_raster_b200.batched``)."""
import os
import sys

from . import _C, meta, renderer, sparse_adam  # noqa: F401

__all__ = ["renderer", "sparse_adam", "meta", "install_as_svraster_cuda"]


def install_as_svraster_cuda():
    """Make ``import svraster_cuda`` resolve to this package (drop-in for the
    reference's training / render loops)."""
    compat = os.path.join(os.path.dirname(os.path.abspath(__file__)), "compat")
    if compat not in sys.path:
        sys.path.insert(0, compat)
    import importlib
    return importlib.import_module("svraster_cuda")
