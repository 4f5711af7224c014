"""Build recipe for ``oracle/_ref``: the reference CUDA backends compiled as checkers.

TEST INFRASTRUCTURE ONLY.  This script compiles the reference's own sources
(``backends/<backend>/src/*.cu`` and ``binding.cpp`` of panicPaul/sv_raster,
read in place from the reference checkout) into one Python extension module
per backend: ``oracle/_ref/svraster_ref_C.so`` (backends/cuda) and
``oracle/_ref/new_svraster_ref_C.so`` (backends/new_cuda, 21-level octrees).  It does not run the
reference's ``setup.py``: it calls ``torch.utils.cpp_extension.load`` with the
source list that ``backends/cuda/setup.py:14-26`` names, for sm_100a, without
fast-math (the reference passes no extra flags, ``setup.py:11-27``).

The built module is used only by ``tests/`` (bit-exact integer parity and FP32
tolerance parity on the GPU) and by the golden-fixture generator
``tests/golden/make_golden.py``.  Nothing in ``sv_raster_b200`` imports it.

The reference checkout is taken from the command line, else from the
SVR_REFERENCE_ROOT environment variable, else from the container's read-only
mount (DEFAULT_ROOT).

Usage:  python oracle/build_ref.py [REFERENCE_ROOT]
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
MODULE = "svraster_ref_C"
# the reference's backends built as checkers: backends/cuda (16-level octrees)
# and backends/new_cuda (21 levels, 128-bit sort keys); same source list
# (setup.py:14-26 of each)
MODULES = {"cuda": "svraster_ref_C", "new_cuda": "new_svraster_ref_C"}
DEFAULT_ROOT = "/root/reference"


def reference_root():
    """Where the reference checkout is read from (None when it is absent)."""
    root = os.environ.get("SVR_REFERENCE_ROOT") or DEFAULT_ROOT
    return root if os.path.isdir(os.path.join(root, "backends", "cuda")) else None

SOURCES = [
    "src/raster_state.cu",
    "src/preprocess.cu",
    "src/forward.cu",
    "src/backward.cu",
    "src/geo_params_gather.cu",
    "src/sh_compute.cu",
    "src/tv_compute.cu",
    "src/utils.cu",
    "src/adam_step.cu",
    "binding.cpp",
]


def built_path(backend="cuda"):
    return os.path.join(OUT_DIR, MODULES[backend] + ".so")


def build(ref_root=None, verbose=False, backend="cuda"):
    ref_root = ref_root or reference_root()
    if ref_root is None:
        raise FileNotFoundError("reference checkout not found (set SVR_REFERENCE_ROOT)")
    module = MODULES[backend]
    src_dir = os.path.join(ref_root, "backends", backend)
    if not os.path.isdir(src_dir):
        raise FileNotFoundError(f"reference backend not found at {src_dir}")
    srcs = [os.path.join(src_dir, s) for s in SOURCES]
    newest_src = max(os.path.getmtime(s) for s in srcs)
    out = built_path(backend)
    if os.path.exists(out) and os.path.getmtime(out) >= newest_src:
        return out
    build_dir = os.path.join(OUT_DIR, "build" if backend == "cuda" else f"build_{backend}")
    os.makedirs(build_dir, exist_ok=True)
    from torch.utils import cpp_extension
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    cpp_extension.load(
        name=module,
        sources=srcs,
        build_directory=build_dir,
        extra_cuda_cflags=["-gencode", "arch=compute_100a,code=sm_100a", "-O3"],
        extra_cflags=["-O3"],
        with_cuda=True,
        is_python_module=True,
        verbose=verbose,
    )
    shutil.copy2(os.path.join(build_dir, module + ".so"), out)
    return out


def load(backend="cuda"):
    """Import the built reference module (no build).  Raises ImportError if absent."""
    import importlib.util
    path = built_path(backend)
    if not os.path.exists(path):
        raise ImportError(f"reference checker module not built: {path}")
    import torch  # noqa: F401  (loads libtorch before the extension)
    spec = importlib.util.spec_from_file_location(MODULES[backend], path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else None
    for b in MODULES:
        print(build(root, verbose=True, backend=b))
