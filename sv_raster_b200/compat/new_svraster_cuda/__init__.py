"""Drop-in stand-in for the reference's ``new_svraster_cuda`` package
(backends/new_cuda, octrees 21 levels deep): put ``sv_raster_b200/compat``
first on ``sys.path`` and ``import new_svraster_cuda`` resolves to
``sv_raster_b200.levels21``."""
import importlib
import sys

_pkg = importlib.import_module("sv_raster_b200.levels21")
for _name in ("_C", "meta", "utils", "renderer", "sparse_adam", "grid_loss_bw"):
    _mod = getattr(_pkg, _name)
    globals()[_name] = _mod
    sys.modules[__name__ + "." + _name] = _mod
