"""Python operator surface of the rasterizer, interface-compatible with
``svraster_cuda.renderer`` (panicPaul/sv_raster, backends/cuda/svraster_cuda/renderer.py).

Same names, argument meanings, return values and exception behaviour; the
native work goes to ``libsvr_b200.so`` through :mod:`sv_raster_b200._C`.
"""
from typing import NamedTuple

import torch

from . import _C


class RasterSettings(NamedTuple):
    """Per-call rasterizer settings (renderer.py:15-36 of the reference)."""
    color_mode: str
    n_samp_per_vox: int
    image_width: int
    image_height: int
    tanfovx: float
    tanfovy: float
    cx: float
    cy: float
    w2c_matrix: torch.Tensor
    c2w_matrix: torch.Tensor
    bg_color: float = 0
    near: float = 0.02
    need_depth: bool = False
    need_normal: bool = False
    track_max_w: bool = False
    lambda_R_concen: float = 0
    lambda_ascending: float = 0
    lambda_dist: float = 0
    gt_color: torch.Tensor = torch.empty(0)
    debug: bool = False


def rasterize_voxels(raster_settings, octree_paths, vox_centers, vox_lengths, vox_fn):
    """Render one view (reference renderer.py:39-127).

    ``vox_fn(visible_idx, cam_pos, color_mode)`` is called between the
    projection pass and compositing and must return a dict with 'geos' [N,8],
    'rgbs' [N,3] and 'subdiv_p' [N,1].  Returns (color, depth, normal, T, max_w).
    """
    s = raster_settings
    if not isinstance(s, RasterSettings):
        raise Exception("Expect RasterSettings as first argument.")
    if s.n_samp_per_vox > _C.MAX_N_SAMP or s.n_samp_per_vox < 1:
        raise Exception(f"n_samp_per_vox should be in range [1, {_C.MAX_N_SAMP}].")
    N = octree_paths.numel()
    device = octree_paths.device
    if vox_centers.shape[0] != N or vox_lengths.numel() != N:
        raise Exception("Size mismatched.")
    if len(vox_centers.shape) != 2 or vox_centers.shape[1] != 3:
        raise Exception("Expect vox_centers in shape [N, 3].")
    for t in (s.w2c_matrix, s.c2w_matrix, vox_centers, vox_lengths):
        if t.device != device:
            raise Exception("Device mismatch.")

    n_duplicates, geom = _C.rasterize_preprocess(
        s.image_width, s.image_height, s.tanfovx, s.tanfovy, s.cx, s.cy, s.w2c_matrix, s.c2w_matrix, s.near,
        octree_paths, vox_centers, vox_lengths, s.debug)
    visible = torch.where(n_duplicates > 0)[0]

    cam_pos = s.c2w_matrix[:3, 3]
    params = vox_fn(visible, cam_pos, s.color_mode)
    geos, rgbs, subdiv_p = params['geos'], params['rgbs'], params['subdiv_p']
    if geos.shape != (N, 8):
        raise Exception(f"Expect geos in ({N}, 8) but got", geos.shape)
    if rgbs.shape[0] != N:
        raise Exception(f"Expect rgbs in ({N}, 3) but got", rgbs.shape)
    if subdiv_p.shape[0] != N:
        raise Exception(f"Expect subdiv_p in ({N}, 1) but got", subdiv_p.shape)
    if geos.device != device:
        raise Exception("Device mismatch: geos.")
    if rgbs.device != device:
        raise Exception("Device mismatch: rgbs.")
    if subdiv_p.device != device:
        raise Exception("Device mismatch: subdiv_p.")
    if s.lambda_R_concen > 0:
        gt = s.gt_color
        if len(gt.shape) != 3 or gt.shape[0] != 3 or gt.shape[1] != s.image_height or gt.shape[2] != s.image_width:
            raise Exception("Except gt_color in shape of [3, H, W]")
        if gt.device != device:
            raise Exception("Device mismatch.")

    return _RasterizeVoxels.apply(s, geom, octree_paths, vox_centers, vox_lengths, geos, rgbs, subdiv_p)


class _RasterizeVoxels(torch.autograd.Function):
    """Compositing with a recompute-transmittance backward (reference renderer.py:130-248)."""

    @staticmethod
    def forward(ctx, raster_settings, geomBuffer, octree_paths, vox_centers, vox_lengths, geos, rgbs, subdiv_p):
        s = raster_settings
        need_distortion = s.lambda_dist > 0
        num_rendered, binning, img, color, depth, normal, T, max_w = _C.rasterize_voxels(
            s.n_samp_per_vox, s.image_width, s.image_height, s.tanfovx, s.tanfovy, s.cx, s.cy, s.w2c_matrix,
            s.c2w_matrix, s.bg_color, s.need_depth, need_distortion, s.need_normal, s.track_max_w, octree_paths,
            vox_centers, vox_lengths, geos, rgbs, geomBuffer, s.debug)
        ctx.raster_settings = s
        ctx.num_rendered = num_rendered
        ctx.save_for_backward(octree_paths, vox_centers, vox_lengths, geos, rgbs, geomBuffer, binning, img, T,
                              depth, normal)
        ctx.mark_non_differentiable(max_w)
        return color, depth, normal, T, max_w

    @staticmethod
    def backward(ctx, dL_dcolor, dL_ddepth, dL_dnormal, dL_dT, dL_dmax_w):
        s = ctx.raster_settings
        (octree_paths, vox_centers, vox_lengths, geos, rgbs, geomBuffer, binning, img, T, depth,
         normal) = ctx.saved_tensors
        dL_dgeos, dL_drgbs, subdiv_p_bw = _C.rasterize_voxels_backward(
            ctx.num_rendered, s.n_samp_per_vox, s.image_width, s.image_height, s.tanfovx, s.tanfovy, s.cx, s.cy,
            s.w2c_matrix, s.c2w_matrix, s.bg_color, octree_paths, vox_centers, vox_lengths, geos, rgbs, geomBuffer,
            binning, img, T, dL_dcolor, dL_ddepth, dL_dnormal, dL_dT, s.lambda_R_concen, s.gt_color,
            s.lambda_ascending, s.lambda_dist, s.need_depth, s.need_normal, depth, normal, s.debug)
        return None, None, None, None, None, dL_dgeos, dL_drgbs, subdiv_p_bw


class SH_eval(torch.autograd.Function):
    """View-dependent colour from SH coefficients (reference renderer.py:251-316)."""

    @staticmethod
    def forward(ctx, active_sh_degree, idx, vox_centers, cam_pos, viewdir, sh0, shs):
        if torch.is_tensor(vox_centers) and vox_centers.requires_grad:
            raise NotImplementedError
        if torch.is_tensor(cam_pos) and cam_pos.requires_grad:
            raise NotImplementedError
        if torch.is_tensor(viewdir) and viewdir.requires_grad:
            raise NotImplementedError
        if idx is None:
            idx = torch.empty(0, dtype=torch.int64)
        if viewdir is not None:
            vox_centers = viewdir
            cam_pos = torch.zeros_like(cam_pos)
        rgbs = _C.sh_compute(active_sh_degree, idx, vox_centers, cam_pos, sh0, shs)
        ctx.active_sh_degree = active_sh_degree
        ctx.M = 1 + shs.shape[1]
        ctx.save_for_backward(idx, vox_centers, cam_pos, rgbs)
        return rgbs

    @staticmethod
    def backward(ctx, dL_drgbs):
        idx, vox_centers, cam_pos, rgbs = ctx.saved_tensors
        dL_dsh0, dL_dshs = _C.sh_compute_bw(ctx.active_sh_degree, ctx.M, idx, vox_centers, cam_pos, rgbs, dL_drgbs)
        return None, None, None, None, None, dL_dsh0, dL_dshs


class GatherGeoParams(torch.autograd.Function):
    """Grid-point densities -> per-voxel 8 corners (reference renderer.py:319-345)."""

    @staticmethod
    def forward(ctx, vox_key, care_idx, grid_pts):
        assert len(vox_key.shape) == 2 and vox_key.shape[1] == 8
        assert len(care_idx.shape) == 1
        assert grid_pts.shape[0] == grid_pts.numel()
        out = _C.gather_triinterp_geo_params(vox_key, care_idx, grid_pts)
        ctx.num_grid_pts = grid_pts.numel()
        ctx.save_for_backward(vox_key, care_idx)
        return out

    @staticmethod
    def backward(ctx, dL_dgeo_params):
        vox_key, care_idx = ctx.saved_tensors
        return None, None, _C.gather_triinterp_geo_params_bw(vox_key, care_idx, ctx.num_grid_pts, dL_dgeo_params)


class GatherFeatParams(torch.autograd.Function):
    """Grid-point 3-vectors -> per-voxel [N,8,3] (reference renderer.py:348-374)."""

    @staticmethod
    def forward(ctx, vox_key, care_idx, grid_pts):
        assert len(vox_key.shape) == 2 and vox_key.shape[1] == 8
        assert len(care_idx.shape) == 1
        assert len(grid_pts.shape) == 2
        out = _C.gather_triinterp_feat_params(vox_key, care_idx, grid_pts)
        ctx.num_grid_pts = len(grid_pts)
        ctx.save_for_backward(vox_key, care_idx)
        return out

    @staticmethod
    def backward(ctx, dL_dfeat_params):
        vox_key, care_idx = ctx.saved_tensors
        return None, None, _C.gather_triinterp_feat_params_bw(vox_key, care_idx, ctx.num_grid_pts, dL_dfeat_params)


def mark_n_duplicates(image_width, image_height, tanfovx, tanfovy, cx, cy, w2c_matrix, c2w_matrix, near,
                      octree_paths, vox_centers, vox_lengths, return_buffer=False, debug=False):
    """Projection pass only (reference renderer.py:377-405)."""
    n_duplicates, geom = _C.rasterize_preprocess(image_width, image_height, tanfovx, tanfovy, cx, cy, w2c_matrix,
                                                 c2w_matrix, near, octree_paths, vox_centers, vox_lengths, debug)
    if return_buffer:
        return n_duplicates, geom
    return n_duplicates


def mark_max_samp_rate(cameras, octree_paths, vox_centers, vox_lengths, near=0.02):
    """Largest sampling rate (voxel size / pixel footprint) over cameras (reference renderer.py:408-423)."""
    max_rate = torch.zeros([len(octree_paths)], dtype=torch.float32, device=vox_centers.device)
    for cam in cameras:
        ndup = mark_n_duplicates(cam.image_width, cam.image_height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy,
                                 cam.w2c, cam.c2w, near, octree_paths, vox_centers, vox_lengths)
        zdist = ((vox_centers - cam.position) * cam.lookat).sum(-1)
        vis = torch.where((ndup > 0) & (zdist > near))[0]
        rate = vox_lengths.squeeze(1)[vis] / (zdist[vis] * cam.pix_size)
        max_rate[vis] = torch.maximum(max_rate[vis], rate)
    return max_rate


def mark_near(cameras, octree_paths, vox_centers, vox_lengths, near=0.2):
    """Voxels within `near` (plus their size) of any camera (reference renderer.py:426-438)."""
    is_near = torch.zeros([len(octree_paths)], dtype=torch.bool, device=vox_centers.device)
    for cam in cameras:
        ndup = mark_n_duplicates(cam.image_width, cam.image_height, cam.tanfovx, cam.tanfovy, cam.cx, cam.cy,
                                 cam.w2c, cam.c2w, near, octree_paths, vox_centers, vox_lengths)
        vis = torch.where(ndup > 0)[0]
        zdist = ((vox_centers[vis] - cam.position) * cam.lookat).sum(-1)
        is_near[vis] |= (zdist <= near + vox_lengths.squeeze(1)[vis])
    return is_near
