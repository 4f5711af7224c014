"""numpy front end of the C oracle (oracle/svr_oracle.c) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() (as the checker) and bench.py's CPU
baseline leg use this module.  ``mode='f32'`` is the fp32 mimic of the GPU
arithmetic, ``mode='f64'`` the FP64 accuracy oracle.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
TILE = 16

_libs = {}


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib(mode):
    if mode not in _libs:
        path = os.path.join(BUILD, f"liboracle_{mode}.so")
        if not os.path.exists(path):
            build()
        _libs[mode] = ctypes.CDLL(path)
    return _libs[mode]


class OrcView(ctypes.Structure):
    _fields_ = [("W", ctypes.c_int), ("H", ctypes.c_int), ("tanfovx", ctypes.c_float), ("tanfovy", ctypes.c_float),
                ("cx", ctypes.c_float), ("cy", ctypes.c_float), ("c2w", ctypes.c_void_p), ("bg", ctypes.c_float),
                ("n_samp", ctypes.c_int), ("need_depth", ctypes.c_int), ("need_dist", ctypes.c_int),
                ("need_normal", ctypes.c_int), ("track_max_w", ctypes.c_int)]


def _p(a):
    return ctypes.c_void_p(0) if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def real_dtype(mode):
    return np.float32 if mode == "f32" else np.float64


def preprocess(cam, centers, lengths, mode="f32"):
    """Returns n_dup u32 [P], bbox u32 [P,2], quad u32 [P] (preprocess.cu:24-132)."""
    P = len(centers)
    ndup = np.zeros(P, np.uint32)
    bbox = np.zeros((P, 2), np.uint32)
    quad = np.zeros(P, np.uint32)
    w2c = _c(cam.w2c, np.float32).reshape(-1)
    c2w = _c(cam.c2w, np.float32).reshape(-1)
    fn = getattr(_lib("f32"), "orc_preprocess_f32")
    fn(ctypes.c_int(P), ctypes.c_int(cam.width), ctypes.c_int(cam.height), ctypes.c_float(cam.tanfovx),
       ctypes.c_float(cam.tanfovy), ctypes.c_float(cam.cx), ctypes.c_float(cam.cy), _p(w2c), _p(c2w),
       ctypes.c_float(cam.near), _p(_c(centers, np.float32)), _p(_c(lengths, np.float32)), _p(ndup), _p(bbox),
       _p(quad))
    return ndup, bbox, quad


def binning(cam, octpath, ndup, bbox, quad):
    """Sorted keys u64 [I], values u32 [I], ranges u32 [T,2] (forward.cu:518-598)."""
    n = int(ndup.astype(np.int64).sum())
    keys = np.zeros(max(n, 1), np.uint64)
    vals = np.zeros(max(n, 1), np.uint32)
    gx, gy = (cam.width + TILE - 1) // TILE, (cam.height + TILE - 1) // TILE
    ranges = np.zeros((gx * gy, 2), np.uint32)
    fn = _lib("f32").orc_binning
    fn.restype = ctypes.c_int64
    got = fn(ctypes.c_int(len(ndup)), ctypes.c_int(cam.width), ctypes.c_int(cam.height),
             _p(_c(octpath, np.int64)), _p(_c(ndup, np.uint32)), _p(_c(bbox, np.uint32)), _p(_c(quad, np.uint32)),
             _p(keys), _p(vals), _p(ranges))
    assert got == n
    return keys[:n], vals[:n], ranges


def _view(cam, n_samp, bg, need_depth, need_dist, need_normal, track_max_w, c2w):
    return OrcView(cam.width, cam.height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy, c2w.ctypes.data, float(bg),
                   n_samp, int(need_depth), int(need_dist), int(need_normal), int(track_max_w))


def render_fwd(cam, ranges, vals, bbox, centers, lengths, geos, rgbs, n_samp=1, bg=0.0, need_depth=False,
               need_dist=False, need_normal=False, track_max_w=False, mode="f32", tiles=None):
    """Forward compositing; returns dict(color [3,H,W], T [H,W], n_contrib [H,W], tile_last [T], ...)."""
    W, H = cam.width, cam.height
    gx, gy = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
    R = real_dtype(mode)
    c2w = _c(cam.c2w, np.float32).reshape(-1)
    v = _view(cam, n_samp, bg, need_depth, need_dist, need_normal, track_max_w, c2w)
    out = dict(color=np.zeros((3, H, W), R), T=np.zeros((H, W), R), n_contrib=np.zeros((H, W), np.uint32),
               tile_last=np.zeros(gx * gy, np.uint32), depth=np.zeros((3, H, W), R), normal=np.zeros((3, H, W), R),
               max_w=np.zeros(len(centers), R))
    fn = getattr(_lib(mode), f"orc_render_fwd_{mode}")
    t0, t1 = (0, gx * gy) if tiles is None else tiles
    fn(ctypes.byref(v), ctypes.c_int(t0), ctypes.c_int(t1), _p(_c(ranges, np.uint32)), _p(_c(vals, np.uint32)),
       _p(_c(bbox, np.uint32)), _p(_c(centers, np.float32)), _p(_c(lengths, np.float32)), _p(_c(geos, np.float32)),
       _p(_c(rgbs, np.float32)), _p(out["tile_last"]), _p(out["n_contrib"]), _p(out["color"]), _p(out["depth"]),
       _p(out["normal"]), _p(out["T"]), _p(out["max_w"]))
    return out


def render_bwd(cam, ranges, tile_last, vals, bbox, centers, lengths, geos, rgbs, n_contrib, T, dL_dcolor, dL_dT,
               n_samp=1, bg=0.0, dL_ddepth=None, dL_dnormal=None, lambda_R=0.0, gt=None, lambda_asc=0.0,
               lambda_dist=0.0, out_depth=None, need_depth=False, need_normal=False, mode="f32", tiles=None):
    """Backward; returns dict(dL_dgeos [P,8], dL_drgbs [P,3], subdiv [P])."""
    W, H = cam.width, cam.height
    gx, gy = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
    R = real_dtype(mode)
    P = len(centers)
    c2w = _c(cam.c2w, np.float32).reshape(-1)
    v = _view(cam, n_samp, bg, need_depth, lambda_dist > 0, need_normal, False, c2w)
    out = dict(dL_dgeos=np.zeros((P, 8), R), dL_drgbs=np.zeros((P, 3), R), subdiv=np.zeros(P, R))
    fn = getattr(_lib(mode), f"orc_render_bwd_{mode}")
    t0, t1 = (0, gx * gy) if tiles is None else tiles
    f32 = lambda a: None if a is None else _c(a, np.float32)
    fn(ctypes.byref(v), ctypes.c_int(t0), ctypes.c_int(t1), _p(_c(ranges, np.uint32)), _p(_c(tile_last, np.uint32)),
       _p(_c(vals, np.uint32)), _p(_c(bbox, np.uint32)), _p(_c(centers, np.float32)), _p(_c(lengths, np.float32)),
       _p(_c(geos, np.float32)), _p(_c(rgbs, np.float32)), _p(_c(n_contrib, np.uint32)), _p(_c(T, R)),
       _p(f32(dL_dcolor)), _p(f32(dL_ddepth)), _p(f32(dL_dnormal)), _p(f32(dL_dT)), ctypes.c_float(lambda_R),
       _p(f32(gt)), ctypes.c_float(lambda_asc), ctypes.c_float(lambda_dist),
       _p(None if out_depth is None else _c(out_depth, R)), _p(out["dL_dgeos"]), _p(out["dL_drgbs"]),
       _p(out["subdiv"]))
    return out


def sh_fwd(deg, idx, centers, campos, sh0, shs, mode="f32"):
    P = len(centers)
    R = real_dtype(mode)
    rgbs = np.zeros((P, 3), R)
    idx = _c(idx, np.int64)
    M = 1 + shs.shape[1]
    getattr(_lib(mode), f"orc_sh_fwd_{mode}")(
        ctypes.c_int(deg), ctypes.c_int(len(idx)), _p(idx), ctypes.c_int(M), _p(_c(centers, np.float32)),
        _p(_c(campos, np.float32)), _p(_c(sh0, np.float32)), _p(_c(shs, np.float32)), _p(rgbs))
    return rgbs


def sh_bwd(deg, M, idx, centers, campos, dL_drgb, mode="f32"):
    P = len(centers)
    R = real_dtype(mode)
    d0 = np.zeros((P, 3), R)
    ds = np.zeros((P, M - 1, 3), R)
    idx = _c(idx, np.int64)
    getattr(_lib(mode), f"orc_sh_bwd_{mode}")(
        ctypes.c_int(deg), ctypes.c_int(len(idx)), _p(idx), ctypes.c_int(M), _p(_c(centers, np.float32)),
        _p(_c(campos, np.float32)), _p(_c(dL_drgb, np.float32)), _p(d0), _p(ds))
    return d0, ds


def adam(param, grad, m, v, step, lr, b1, b2, eps, biased=False, sparse=False, mode="f32"):
    """In-place Adam on REAL arrays param/m/v (copies returned)."""
    R = real_dtype(mode)
    p, mm, vv = _c(param, R).copy(), _c(m, R).copy(), _c(v, R).copy()
    getattr(_lib(mode), f"orc_adam_{mode}")(
        ctypes.c_int(int(biased)), ctypes.c_int(int(sparse)), ctypes.c_int64(p.size), _p(p), _p(_c(grad, np.float32)),
        _p(mm), _p(vv), ctypes.c_double(step), ctypes.c_double(lr), ctypes.c_double(b1), ctypes.c_double(b2),
        ctypes.c_float(eps))
    return p, mm, vv


def render_view(cam, octpath, centers, lengths, geos, rgbs, n_samp=1, bg=0.0, mode="f32", **flags):
    """Preprocess + binning + forward for one camera."""
    ndup, bbox, quad = preprocess(cam, centers, lengths)
    keys, vals, ranges = binning(cam, octpath, ndup, bbox, quad)
    out = render_fwd(cam, ranges, vals, bbox, centers, lengths, geos, rgbs, n_samp=n_samp, bg=bg, mode=mode,
                     **flags)
    out.update(ndup=ndup, bbox=bbox, quad=quad, keys=keys, vals=vals, ranges=ranges)
    return out
