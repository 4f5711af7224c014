"""Build ``libsvr_b200.so`` (all CUDA kernels + the C ABI) in-tree for sm_100a.

Each ``csrc/*.cu`` file is compiled by nvcc in parallel with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` (default FMA
contraction, no fast-math: the same floating-point mode as the reference
backend build) and linked into ``sv_raster_b200/libsvr_b200.so`` with the CUDA
runtime linked statically, so the library does not depend on which libcudart
the host process loaded.  Rebuilds only what changed (mtime of sources and
headers).

Usage: python -m sv_raster_b200.build [--force] [--verbose]
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libsvr_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                     "--expt-relaxed-constexpr", "-I", CSRC, "-I", INCLUDE]


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; set NVCC or install the CUDA toolkit")
    return cand


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _compile(src, obj, verbose):
    cmd = [nvcc(), "-c", src, "-o", obj] + NVCC_FLAGS
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force=False, verbose=False):
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    newest_src = max([os.path.getmtime(s) for s in srcs] + [hdr_mtime])
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest_src:
        return LIB  # up to date (object files need not be present)
    os.makedirs(OBJ, exist_ok=True)
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_mtime):
            jobs.append((s, o))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(lambda j: _compile(j[0], j[1], verbose), jobs))
    newest_obj = max(os.path.getmtime(o) for o in objs)
    if force or jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest_obj:
        tmp = LIB + ".tmp"
        cmd = [nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-cudart", "static", "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
