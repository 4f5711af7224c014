"""Build recipe for ``oracle/_ref``: the reference CUDA backend compiled as a checker.

TEST INFRASTRUCTURE ONLY.  This script compiles the reference's own sources
(``backends/cuda/src/*.cu`` and ``backends/cuda/binding.cpp`` of
panicPaul/sv_raster, read in place from the reference checkout) into a single
Python extension module ``oracle/_ref/svraster_ref_C.so``.  It does not run the
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


def built_path():
    return os.path.join(OUT_DIR, MODULE + ".so")


def build(ref_root=None, verbose=False):
    ref_root = ref_root or reference_root()
    if ref_root is None:
        raise FileNotFoundError("reference checkout not found (set SVR_REFERENCE_ROOT)")
    backend = os.path.join(ref_root, "backends", "cuda")
    if not os.path.isdir(backend):
        raise FileNotFoundError(f"reference backend not found at {backend}")
    srcs = [os.path.join(backend, s) for s in SOURCES]
    newest_src = max(os.path.getmtime(s) for s in srcs)
    if os.path.exists(built_path()) and os.path.getmtime(built_path()) >= newest_src:
        return built_path()
    build_dir = os.path.join(OUT_DIR, "build")
    os.makedirs(build_dir, exist_ok=True)
    from torch.utils import cpp_extension
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    cpp_extension.load(
        name=MODULE,
        sources=srcs,
        build_directory=build_dir,
        extra_cuda_cflags=["-gencode", "arch=compute_100a,code=sm_100a", "-O3"],
        extra_cflags=["-O3"],
        with_cuda=True,
        is_python_module=True,
        verbose=verbose,
    )
    shutil.copy2(os.path.join(build_dir, MODULE + ".so"), built_path())
    return built_path()


def load():
    """Import the built reference module (no build).  Raises ImportError if absent."""
    import importlib.util
    path = built_path()
    if not os.path.exists(path):
        raise ImportError(f"reference checker module not built: {path}")
    import torch  # noqa: F401  (loads libtorch before the extension)
    spec = importlib.util.spec_from_file_location(MODULE, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else None, verbose=True))
