"""Total-variation gradient on grid points, interface of
``svraster_cuda.grid_loss_bw`` (backends/cuda/svraster_cuda/grid_loss_bw.py)."""
import ctypes

import torch

from ._native import check, lib


def total_variation(grid_pts, vox_key, weight, vox_size_inv, no_tv_s, tv_sparse, grid_pts_grad):
    """Adds the TV gradient into ``grid_pts_grad`` in place (tv_compute.cu:84-110)."""
    assert grid_pts.shape == grid_pts_grad.shape
    assert len(vox_key.shape) == 2 and vox_key.shape[1] == 8
    assert vox_key.shape[0] == vox_size_inv.numel()
    if not grid_pts_grad.is_contiguous():
        raise RuntimeError("grid_pts_grad must be contiguous (updated in place)")
    N = vox_key.shape[0]
    C = grid_pts.shape[1] if grid_pts.dim() > 1 else 1
    dev = grid_pts.device
    g = grid_pts.contiguous().float()
    k = vox_key.contiguous().to(torch.int64)
    s = vox_size_inv.contiguous().float()
    scratch = torch.empty(N * C, dtype=torch.uint8, device=dev) if tv_sparse else None
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
    with torch.cuda.device(dev):
        st = lib().svr_total_variation_bw(p(g), p(k), float(weight), p(s), int(bool(no_tv_s)), int(bool(tv_sparse)),
                                          N, C, p(scratch), p(grid_pts_grad),
                                          ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    check(st, "total_variation_bw")
