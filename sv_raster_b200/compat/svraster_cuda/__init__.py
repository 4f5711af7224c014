"""Drop-in stand-in for the reference's ``svraster_cuda`` package.

Put ``sv_raster_b200/compat`` first on ``sys.path`` (or
``sv_raster_b200.install_as_svraster_cuda()``) and the reference's training
and render loops (``import svraster_cuda``; ``svraster_cuda.renderer...``)
run on the sm_100a kernels unchanged.
"""
import importlib
import sys

_pkg = importlib.import_module("sv_raster_b200")
_C = importlib.import_module("sv_raster_b200._C")
meta = importlib.import_module("sv_raster_b200.meta")
utils = importlib.import_module("sv_raster_b200.utils")
renderer = importlib.import_module("sv_raster_b200.renderer")
sparse_adam = importlib.import_module("sv_raster_b200.sparse_adam")
grid_loss_bw = importlib.import_module("sv_raster_b200.grid_loss_bw")

for _name, _mod in (("_C", _C), ("meta", meta), ("utils", utils), ("renderer", renderer),
                    ("sparse_adam", sparse_adam), ("grid_loss_bw", grid_loss_bw)):
    sys.modules[__name__ + "." + _name] = _mod
