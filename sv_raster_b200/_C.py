"""Native op surface with the signatures of the reference's pybind11 module.

Every function here has the name, argument order, return structure and
zero-initialisation behaviour of the corresponding export of
``svraster_cuda._C`` (panicPaul/sv_raster, backends/cuda/binding.cpp:24-55),
so ``renderer.py`` / ``sparse_adam.py`` read like the reference's.  Outputs
are allocated with torch on the inputs' device and handed to
``libsvr_b200.so`` as raw pointers together with the current CUDA stream.
"""
import ctypes

import torch

from . import _native
from ._native import Camera, check, lib

MAX_NUM_LEVELS = 16   # config.h:16
STEP_SZ_SCALE = 100.0  # config.h:21
MAX_N_SAMP = 3         # config.h:23

TILE = 16


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if (t is not None and t.numel() > 0) else ctypes.c_void_p(0)


def _stream(dev):
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _f32(t, name):
    if t.dtype != torch.float32:
        raise RuntimeError(f"{name}: expected scalar type Float but found {t.dtype}")
    return t.contiguous()


def _i64(t, name):
    if t.dtype != torch.int64:
        raise RuntimeError(f"{name}: expected scalar type Long but found {t.dtype}")
    return t.contiguous()


def _cuda(t, name):
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    return t


def _camera(W, H, tanfovx, tanfovy, cx, cy, w2c, c2w, near=0.02, bg=0.0):
    return Camera(int(W), int(H), float(tanfovx), float(tanfovy), float(cx), float(cy),
                  w2c.data_ptr(), c2w.data_ptr(), float(near), float(bg))


def _mat(t, name, dev):
    t = _f32(t, name)
    if t.numel() < 12:
        raise RuntimeError(f"{name} must hold a 4x4 (or 3x4) matrix")
    return _cuda(t, name).to(dev)


def rasterize_preprocess(image_width, image_height, tan_fovx, tan_fovy, cx, cy, w2c_matrix, c2w_matrix, near,
                         octree_paths, vox_centers, vox_lengths, debug=False):
    """preprocess.cu:136-199 -> (out_n_duplicates int32 [P], geomBuffer uint8)."""
    if vox_centers.ndimension() != 2 or vox_centers.size(1) != 3:
        raise RuntimeError("vox_centers must have dimensions (num_points, 3)")
    dev = _cuda(vox_centers, "vox_centers").device
    P = vox_centers.size(0)
    out_ndup = torch.zeros(P, dtype=torch.int32, device=dev)
    if P == 0:
        return out_ndup, torch.empty(0, dtype=torch.uint8, device=dev)
    L = lib()
    with torch.cuda.device(dev):
        vc = _f32(vox_centers, "vox_centers")
        vl = _f32(vox_lengths, "vox_lengths")
        w2c = _mat(w2c_matrix, "w2c_matrix", dev)
        c2w = _mat(c2w_matrix, "c2w_matrix", dev)
        nbytes = L.svr_geom_buffer_bytes(P)
        geom = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        cam = _camera(image_width, image_height, tan_fovx, tan_fovy, cx, cy, w2c, c2w, near)
        st = L.svr_rasterize_preprocess(ctypes.byref(cam), P, _ptr(octree_paths), _ptr(vc), _ptr(vl), _ptr(out_ndup),
                                        _ptr(geom), nbytes, int(bool(debug)), _stream(dev))
        check(st, "rasterize_preprocess")
        if debug:
            _check_device_error(geom, dev)
    return out_ndup, geom


def _check_device_error(geom, dev):
    word = ctypes.c_uint32(0)
    err_ptr = lib().svr_geom_error_ptr(_ptr(geom))
    st = lib().svr_read_error(ctypes.c_void_p(err_ptr), ctypes.byref(word), _stream(dev))
    if st != 0:
        raise RuntimeError(f"device consistency check failed (error word 0x{word.value:x})")


def geom_num_rendered(geomBuffer):
    """Instance count left in a geom buffer by rasterize_preprocess (host sync)."""
    if geomBuffer.numel() == 0:
        return 0
    return int(geomBuffer[:4].view(torch.int32).item()) & 0xFFFFFFFF


def rasterize_voxels(n_samp_per_vox, image_width, image_height, tan_fovx, tan_fovy, cx, cy, w2c_matrix, c2w_matrix,
                     bg_color, need_depth, need_distortion, need_normal, track_max_w, octree_paths, vox_centers,
                     vox_lengths, geos, rgbs, geomBuffer, debug=False, levels=MAX_NUM_LEVELS):
    """forward.cu:739-825 -> (num_rendered, binningBuffer, imgBuffer, color, depth, normal, T, max_w).
    ``levels`` = 21 bins octrees 21 levels deep (the new_cuda backend's forward)."""
    if vox_centers.ndimension() != 2 or vox_centers.size(1) != 3:
        raise RuntimeError("vox_centers must have dimensions (num_points, 3)")
    if rgbs.ndimension() != 2 or rgbs.size(1) != 3:
        raise RuntimeError("rgbs should be either (num_points, 3)")
    if vox_centers.size(0) != rgbs.size(0):
        raise RuntimeError("size mismatch")
    dev = _cuda(vox_centers, "vox_centers").device
    P = vox_centers.size(0)
    H, W = int(image_height), int(image_width)
    fopt = dict(dtype=torch.float32, device=dev)
    color = torch.zeros(3, H, W, **fopt)
    depth = torch.zeros(3, H, W, **fopt) if (need_depth or need_distortion) else torch.empty(0)
    normal = torch.zeros(3, H, W, **fopt) if need_normal else torch.empty(0)
    T = torch.zeros(1, H, W, **fopt)
    max_w = torch.zeros(P, 1, **fopt) if track_max_w else torch.empty(0)
    binning = torch.empty(0, dtype=torch.uint8, device=dev)
    L = lib()
    img = torch.empty(L.svr_image_buffer_bytes(W, H), dtype=torch.uint8, device=dev)
    if P == 0:
        return 0, binning, img, color, depth, normal, T, max_w
    with torch.cuda.device(dev):
        num_rendered = geom_num_rendered(geomBuffer)  # host sync, as forward.cu:653
        if num_rendered == 0xFFFFFFFF:
            raise RuntimeError("rasterize_voxels: instance count overflows 32 bits")
        if levels == MAX_NUM_LEVELS:
            nbytes = L.svr_binning_buffer_bytes(num_rendered, W, H)
        else:
            nbytes = L.svr_binning_buffer_bytes_levels(num_rendered, W, H, int(levels))
            if nbytes == 0:
                raise RuntimeError(f"rasterize_voxels: unsupported octree depth {levels}")
        binning = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        op = _i64(octree_paths, "octree_paths").reshape(-1)
        vc = _f32(vox_centers, "vox_centers")
        vl = _f32(vox_lengths, "vox_lengths")
        g = _f32(geos, "geos")
        c = _f32(rgbs, "rgbs")
        w2c = _mat(w2c_matrix, "w2c_matrix", dev)
        c2w = _mat(c2w_matrix, "c2w_matrix", dev)
        cam = _camera(W, H, tan_fovx, tan_fovy, cx, cy, w2c, c2w, 0.02, bg_color)
        head = (ctypes.byref(cam), int(n_samp_per_vox), int(bool(need_depth)), int(bool(need_distortion)),
                int(bool(need_normal)), int(bool(track_max_w)), P, num_rendered, _ptr(op))
        fwd = L.svr_rasterize_forward if levels == MAX_NUM_LEVELS else \
            (lambda *a: L.svr_rasterize_forward_levels(*a[:9], int(levels), *a[9:]))
        st = fwd(
            *head, _ptr(vc), _ptr(vl), _ptr(g), _ptr(c), _ptr(geomBuffer),
            _ptr(binning), binning.numel(), _ptr(img), img.numel(),
            _ptr(color), _ptr(depth) if (need_depth or need_distortion) else None,
            _ptr(normal) if need_normal else None, _ptr(T), _ptr(max_w) if track_max_w else None,
            int(bool(debug)), _stream(dev))
        check(st, "rasterize_voxels")
        if debug:
            _check_device_error(geomBuffer, dev)
    return num_rendered, binning, img, color, depth, normal, T, max_w


def rasterize_voxels_backward(R, n_samp_per_vox, image_width, image_height, tan_fovx, tan_fovy, cx, cy, w2c_matrix,
                              c2w_matrix, bg_color, octree_paths, vox_centers, vox_lengths, geos, rgbs, geomBuffer,
                              binningBuffer, imageBuffer, out_T, dL_dout_color, dL_dout_depth, dL_dout_normal,
                              dL_dout_T, lambda_R_concen, gt_color, lambda_ascending, lambda_dist, need_depth,
                              need_normal, out_D, out_N, debug=False):
    """backward.cu:655-769 -> (dL_dgeos [P,8], dL_drgbs [P,3], subdiv_p_bw [P,1])."""
    if vox_centers.ndimension() != 2 or vox_centers.size(1) != 3:
        raise RuntimeError("vox_centers must have dimensions (num_points, 3)")
    dev = _cuda(vox_centers, "vox_centers").device
    P = vox_centers.size(0)
    if P == 0:
        e = torch.empty(0)
        return e, e.clone(), e.clone()
    H, W = int(image_height), int(image_width)
    fopt = dict(dtype=torch.float32, device=dev)
    dL_dgeos = torch.zeros(P, geos.size(1), **fopt)
    dL_drgbs = torch.zeros(P, 3, **fopt)
    subdiv = torch.zeros(P, 1, **fopt)
    need_dist = lambda_dist > 0
    L = lib()
    with torch.cuda.device(dev):
        vc = _f32(vox_centers, "vox_centers")
        vl = _f32(vox_lengths, "vox_lengths")
        g = _f32(geos, "geos")
        c = _f32(rgbs, "rgbs")
        oT = _f32(out_T, "out_T")
        dC = _f32(dL_dout_color, "dL_dout_color")
        dT = _f32(dL_dout_T, "dL_dout_T")
        dD = _f32(dL_dout_depth, "dL_dout_depth") if need_depth else None
        dN = _f32(dL_dout_normal, "dL_dout_normal") if need_normal else None
        gt = _f32(gt_color, "gt_color") if lambda_R_concen > 0 else None
        oD = _f32(out_D, "out_D") if need_dist else None
        w2c = _mat(w2c_matrix, "w2c_matrix", dev)
        c2w = _mat(c2w_matrix, "c2w_matrix", dev)
        cam = _camera(W, H, tan_fovx, tan_fovy, cx, cy, w2c, c2w, 0.02, bg_color)
        st = L.svr_rasterize_backward(
            ctypes.byref(cam), int(n_samp_per_vox), P, int(R), _ptr(vc), _ptr(vl), _ptr(g), _ptr(c),
            _ptr(geomBuffer), _ptr(binningBuffer), _ptr(imageBuffer), _ptr(oT), _ptr(dC), _ptr(dD), _ptr(dN),
            _ptr(dT), float(lambda_R_concen), _ptr(gt), float(lambda_ascending), float(lambda_dist),
            int(bool(need_depth)), int(bool(need_normal)), _ptr(oD), None, _ptr(dL_dgeos), _ptr(dL_drgbs),
            _ptr(subdiv), int(bool(debug)), _stream(dev))
        check(st, "rasterize_voxels_backward")
        if debug:
            _check_device_error(geomBuffer, dev)
    return dL_dgeos, dL_drgbs, subdiv


def unpack_ImageState(image_width, image_height, imageBuffer):
    """raster_state.cu:155-175 -> (ranges [ty,tx,2], tile_last [ty,tx], n_contrib [H,W]) int32."""
    W, H = int(image_width), int(image_height)
    tx, ty = (W + TILE - 1) // TILE, (H + TILE - 1) // TILE
    dev = imageBuffer.device
    ranges = torch.zeros(ty, tx, 2, dtype=torch.int32, device=dev)
    tile_last = torch.zeros(ty, tx, dtype=torch.int32, device=dev)
    n_contrib = torch.zeros(H, W, dtype=torch.int32, device=dev)
    with torch.cuda.device(dev):
        st = lib().svr_unpack_image_state(W, H, _ptr(imageBuffer), _ptr(ranges), _ptr(tile_last), _ptr(n_contrib),
                                          _stream(dev))
    check(st, "unpack_ImageState")
    return ranges, tile_last, n_contrib


def unpack_sorted_list(binningBuffer, num_rendered, image_width, image_height):
    """Sorted (key, value) arrays of a binning buffer as int64 / int32 tensors (copies)."""
    dev = binningBuffer.device
    if num_rendered == 0:
        return torch.empty(0, dtype=torch.int64, device=dev), torch.empty(0, dtype=torch.int32, device=dev)
    kp, vp = ctypes.c_void_p(), ctypes.c_void_p()
    check(lib().svr_binning_sorted(_ptr(binningBuffer), num_rendered, image_width, image_height,
                                   ctypes.byref(kp), ctypes.byref(vp)), "binning_sorted")
    base = binningBuffer.data_ptr()
    ko, vo = kp.value - base, vp.value - base
    keys = binningBuffer[ko:ko + 8 * num_rendered].view(torch.int64).clone()
    vals = binningBuffer[vo:vo + 4 * num_rendered].view(torch.int32).clone()
    return keys, vals


def unpack_sorted_list_wide(binningBuffer, num_rendered, image_width, image_height):
    """Sorted 128-bit keys (as int64 high and low words) and values of a
    21-level binning buffer (copies)."""
    dev = binningBuffer.device
    if num_rendered == 0:
        e = torch.empty(0, dtype=torch.int64, device=dev)
        return e, e.clone(), torch.empty(0, dtype=torch.int32, device=dev)
    lo, hi, vp = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    check(lib().svr_binning_sorted_wide(_ptr(binningBuffer), num_rendered, image_width, image_height,
                                        ctypes.byref(lo), ctypes.byref(hi), ctypes.byref(vp)), "binning_sorted_wide")
    base = binningBuffer.data_ptr()
    cut = lambda p, n, dt: binningBuffer[p.value - base:p.value - base + n * num_rendered].view(dt).clone()
    return cut(hi, 8, torch.int64), cut(lo, 8, torch.int64), cut(vp, 4, torch.int32)


def unpack_geom_state(geomBuffer, P):
    """(n_dup, scan, bboxes as int64 pairs, quadrant bitsets) of a geom buffer (copies)."""
    if P == 0:
        z = torch.empty(0, dtype=torch.int32)
        return z, z, z, z
    ptrs = [ctypes.c_void_p() for _ in range(4)]
    check(lib().svr_geom_arrays(_ptr(geomBuffer), P, *[ctypes.byref(p) for p in ptrs]), "geom_arrays")
    base = geomBuffer.data_ptr()
    o = [p.value - base for p in ptrs]
    ndup = geomBuffer[o[0]:o[0] + 4 * P].view(torch.int32).clone()
    scan = geomBuffer[o[1]:o[1] + 4 * P].view(torch.int32).clone()
    bbox = geomBuffer[o[2]:o[2] + 8 * P].view(torch.int32).view(P, 2).clone()
    quad = geomBuffer[o[3]:o[3] + 4 * P].view(torch.int32).clone()
    return ndup, scan, bbox, quad


def sh_compute(D, indices, vox_centers, cam_pos, sh0, shs):
    """sh_compute.cu:244-270 -> rgbs [P,3] (zeros outside `indices`)."""
    dev = _cuda(vox_centers, "vox_centers").device
    P = vox_centers.size(0)
    N = indices.size(0) if indices is not None else 0
    M = 1 + shs.size(1)
    rgbs = torch.zeros(P, 3, dtype=torch.float32, device=dev)
    if P == 0:
        return rgbs
    with torch.cuda.device(dev):
        vc = _f32(vox_centers, "vox_centers")
        cp = _f32(cam_pos, "cam_pos").to(dev)
        bf16 = sh0.dtype == torch.bfloat16
        s0 = sh0.contiguous() if bf16 else _f32(sh0, "sh0")
        s = shs.contiguous() if bf16 else _f32(shs, "shs")
        if bf16 and s.dtype != torch.bfloat16:
            raise RuntimeError("sh0 and shs must share a dtype")
        idx = _i64(indices, "indices").to(dev) if N > 0 else None
        st = lib().svr_sh_compute(int(D), N, _ptr(idx), P, M, _ptr(vc), _ptr(cp), _ptr(s0), _ptr(s), int(bf16),
                                  _ptr(rgbs), _stream(dev))
    check(st, "sh_compute")
    return rgbs


def sh_compute_bw(D, M, indices, vox_centers, cam_pos, rgbs, dL_drgbs):
    """sh_compute.cu:272-299 -> (dL_dsh0 [P,3], dL_dshs [P,M-1,3])."""
    dev = _cuda(vox_centers, "vox_centers").device
    P = vox_centers.size(0)
    N = indices.size(0) if indices is not None else 0
    dL_dsh0 = torch.zeros(P, 3, dtype=torch.float32, device=dev)
    dL_dshs = torch.zeros(P, M - 1, 3, dtype=torch.float32, device=dev)
    if P == 0:
        return dL_dsh0, dL_dshs
    with torch.cuda.device(dev):
        vc = _f32(vox_centers, "vox_centers")
        cp = _f32(cam_pos, "cam_pos").to(dev)
        g = _f32(dL_drgbs, "dL_drgbs")
        idx = _i64(indices, "indices").to(dev) if N > 0 else None
        st = lib().svr_sh_compute_bw(int(D), int(M), N, _ptr(idx), P, _ptr(vc), _ptr(cp), _ptr(g), _ptr(dL_dsh0),
                                     _ptr(dL_dshs), _stream(dev))
    check(st, "sh_compute_bw")
    return dL_dsh0, dL_dshs


def _adam_tensors(param, grad, exp_avg, exp_avg_sq):
    for t, n in ((param, "param"), (grad, "grad"), (exp_avg, "exp_avg"), (exp_avg_sq, "exp_avg_sq")):
        if t.dtype != torch.float32:
            raise RuntimeError(f"{n}: expected scalar type Float but found {t.dtype}")
        if not t.is_contiguous():
            raise RuntimeError(f"{n} must be contiguous (updated in place)")
        _cuda(t, n)


def unbiased_adam_step(sparse, param, grad, exp_avg, exp_avg_sq, step, lr, beta1, beta2, eps):
    """adam_step.cu:106-135 (in place)."""
    _adam_tensors(param, grad, exp_avg, exp_avg_sq)
    dev = param.device
    with torch.cuda.device(dev):
        st = lib().svr_unbiased_adam_step(int(bool(sparse)), param.numel(), _ptr(param), _ptr(grad), _ptr(exp_avg),
                                          _ptr(exp_avg_sq), float(step), float(lr), float(beta1), float(beta2),
                                          float(eps), _stream(dev))
    check(st, "unbiased_adam_step")


def biased_adam_step(sparse, param, grad, exp_avg, exp_avg_sq, lr, beta1, beta2, eps):
    """adam_step.cu:137-158 (in place)."""
    _adam_tensors(param, grad, exp_avg, exp_avg_sq)
    dev = param.device
    with torch.cuda.device(dev):
        st = lib().svr_biased_adam_step(int(bool(sparse)), param.numel(), _ptr(param), _ptr(grad), _ptr(exp_avg),
                                        _ptr(exp_avg_sq), float(lr), float(beta1), float(beta2), float(eps),
                                        _stream(dev))
    check(st, "biased_adam_step")


def gather_triinterp_geo_params(vox_key, care_idx, grid_pts):
    """geo_params_gather.cu:134-152 -> geo_params [N,8] (rows outside care_idx uninitialised)."""
    dev = _cuda(grid_pts, "grid_pts").device
    n_vox = vox_key.size(0)
    out = torch.empty(n_vox, 8, dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        st = lib().svr_gather_grid_params(1, care_idx.size(0), _ptr(_i64(vox_key, "vox_key")),
                                          _ptr(_i64(care_idx, "care_idx")), _ptr(_f32(grid_pts, "grid_pts")),
                                          _ptr(out), _stream(dev))
    check(st, "gather_triinterp_geo_params")
    return out


def gather_triinterp_geo_params_bw(vox_key, care_idx, num_grid_pts, dL_dgeo_params):
    """geo_params_gather.cu:154-172 -> dL_dgrid_pts [M,1]."""
    dev = _cuda(dL_dgeo_params, "dL_dgeo_params").device
    out = torch.zeros(int(num_grid_pts), 1, dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        st = lib().svr_gather_grid_params_bw(1, care_idx.size(0), _ptr(_i64(vox_key, "vox_key")),
                                             _ptr(_i64(care_idx, "care_idx")),
                                             _ptr(_f32(dL_dgeo_params, "dL_dgeo_params")), _ptr(out), _stream(dev))
    check(st, "gather_triinterp_geo_params_bw")
    return out


def gather_triinterp_feat_params(vox_key, care_idx, grid_pts):
    """geo_params_gather.cu:174-197 -> feat_params [N,8,3]."""
    if grid_pts.size(1) != 3:
        raise RuntimeError("Only support n_dim=3 now.")
    dev = _cuda(grid_pts, "grid_pts").device
    out = torch.empty(vox_key.size(0), 8, 3, dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        st = lib().svr_gather_grid_params(3, care_idx.size(0), _ptr(_i64(vox_key, "vox_key")),
                                          _ptr(_i64(care_idx, "care_idx")), _ptr(_f32(grid_pts, "grid_pts")),
                                          _ptr(out), _stream(dev))
    check(st, "gather_triinterp_feat_params")
    return out


def gather_triinterp_feat_params_bw(vox_key, care_idx, num_grid_pts, dL_dfeat_params):
    """geo_params_gather.cu:199-222 -> dL_dgrid_pts [M,3]."""
    if dL_dfeat_params.size(2) != 3:
        raise RuntimeError("Only support n_dim=3")
    dev = _cuda(dL_dfeat_params, "dL_dfeat_params").device
    out = torch.zeros(int(num_grid_pts), 3, dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        st = lib().svr_gather_grid_params_bw(3, care_idx.size(0), _ptr(_i64(vox_key, "vox_key")),
                                             _ptr(_i64(care_idx, "care_idx")),
                                             _ptr(_f32(dL_dfeat_params, "dL_dfeat_params")), _ptr(out),
                                             _stream(dev))
    check(st, "gather_triinterp_feat_params_bw")
    return out
