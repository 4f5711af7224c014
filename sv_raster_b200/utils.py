"""Setup / geometry utilities with the interface of ``svraster_cuda.utils``
(backends/cuda/svraster_cuda/utils.py, kernels in backends/cuda/src/utils.cu:23-189).

These run once per scene or per camera, not per pixel, so they are written
with torch tensor operations on the inputs' device.
"""
import torch

from . import _C

MAX_NUM_LEVELS = _C.MAX_NUM_LEVELS  # 16, or 21 for the new_cuda surface (levels21)


def _order_tables(device):
    t = []
    for q in range(8):
        v = 0
        for _ in range(MAX_NUM_LEVELS):
            v = (v << 3) | q
        t.append(v)
    return torch.tensor(t, dtype=torch.int64, device=device)


def voxel_order_rank(octree_paths):
    """[8, P] direction-dependent Morton ranks: octpath ^ repeat(q) (utils.cu:106-127)."""
    p = octree_paths.reshape(-1).to(torch.int64)
    return p[None, :] ^ _order_tables(p.device)[:, None]


def is_in_cone(pts, cam):
    """Points strictly in front of `near` and inside the camera's field of view (utils.cu:23-44)."""
    assert torch.is_tensor(pts)
    assert pts.device == cam.w2c.device
    assert len(pts.shape) == 2 and pts.shape[1] == 3
    w2c = cam.w2c.reshape(-1)[:12].view(3, 4).to(pts.dtype)
    pc = pts @ w2c[:, :3].T + w2c[:, 3]
    return (pc[:, 2] > cam.near) & (pc[:, 0].abs() <= cam.tanfovx * pc[:, 2]) & \
        (pc[:, 1].abs() <= cam.tanfovy * pc[:, 2])


def _cam_dirs(width, height, cx, cy, tanfovx, tanfovy, c2w_matrix):
    dev = c2w_matrix.device
    ys, xs = torch.meshgrid(torch.arange(height, device=dev, dtype=torch.float32),
                            torch.arange(width, device=dev, dtype=torch.float32), indexing="ij")
    dx = (xs + 0.5 - cx) * 2.0 * tanfovx / float(width)
    dy = (ys + 0.5 - cy) * 2.0 * tanfovy / float(height)
    m = c2w_matrix.reshape(-1)[:12].view(3, 4).float()
    d = torch.stack([dx, dy, torch.ones_like(dx)], 0)  # [3,H,W]
    return torch.einsum("ij,jhw->ihw", m[:, :3], d), m[:, 3]


def compute_rd(width, height, cx, cy, tanfovx, tanfovy, c2w_matrix):
    """Unnormalised world ray directions [3,H,W] (utils.cu:46-73)."""
    assert torch.is_tensor(c2w_matrix)
    rd, _ = _cam_dirs(width, height, cx, cy, tanfovx, tanfovy, c2w_matrix)
    return rd


def depth2pts(width, height, cx, cy, tanfovx, tanfovy, c2w_matrix, depth):
    """World points [3,H,W] = origin + depth * unnormalised direction (utils.cu:75-104)."""
    assert torch.is_tensor(c2w_matrix)
    assert depth.device == c2w_matrix.device
    assert depth.numel() == width * height
    rd, o = _cam_dirs(width, height, cx, cy, tanfovx, tanfovy, c2w_matrix)
    return o[:, None, None] + depth.reshape(1, height, width) * rd


def ijk_2_octpath(ijk, octlevel):
    """Cell coordinates at each voxel's level -> octree path [P,1] (utils.cu:129-158)."""
    assert torch.is_tensor(ijk) and torch.is_tensor(octlevel)
    assert len(ijk.shape) == 2 and ijk.shape[1] == 3
    assert ijk.numel() == octlevel.numel() * 3
    assert ijk.dtype == torch.int64
    assert octlevel.dtype == torch.int8
    i, j, k = ijk[:, 0].clone(), ijk[:, 1].clone(), ijk[:, 2].clone()
    path = torch.zeros_like(i)
    for l in range(MAX_NUM_LEVELS):
        path |= (((i & 1) << 2) | ((j & 1) << 1) | (k & 1)) << (3 * l)
        i, j, k = i >> 1, j >> 1, k >> 1
    lv = octlevel.reshape(-1).to(torch.int64)
    return (path << (3 * (MAX_NUM_LEVELS - lv))).reshape(-1, 1)


def octpath_2_ijk(octpath, octlevel):
    """Octree path -> cell coordinates [P,3] (utils.cu:160-189)."""
    assert torch.is_tensor(octpath) and torch.is_tensor(octlevel)
    assert octpath.numel() == octlevel.numel()
    assert octpath.dtype == torch.int64
    assert octlevel.dtype == torch.int8
    lv = octlevel.reshape(-1).to(torch.int64)
    p = octpath.reshape(-1) >> (3 * (MAX_NUM_LEVELS - lv))
    ijk = torch.zeros(p.shape[0], 3, dtype=torch.int64, device=p.device)
    for l in range(MAX_NUM_LEVELS):
        b = p & 7
        ijk[:, 0] |= ((b >> 2) & 1) << l
        ijk[:, 1] |= ((b >> 1) & 1) << l
        ijk[:, 2] |= (b & 1) << l
        p = p >> 3
    return ijk
