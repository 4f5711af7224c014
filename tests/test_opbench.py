"""The operator benchmark's grid builder (CPU): corner indices of octree voxels
into a deduplicated grid address one point per distinct corner position."""
import numpy as np
import torch

from sv_raster_b200 import synthetic
from sv_raster_b200.opbench import grid_keys


def test_grid_keys_share_coincident_corners():
    sc = synthetic.config_scene("c1", n_voxels=3000)
    key, M = grid_keys(sc.octpath, sc.octlevel, torch.device("cpu"))
    assert key.shape == (len(sc.octpath), 8) and int(key.min()) == 0 and int(key.max()) == M - 1
    c = torch.from_numpy(sc.centers).double()
    l = torch.from_numpy(sc.lengths).double()
    off = torch.tensor([[(q >> 2) & 1, (q >> 1) & 1, q & 1] for q in range(8)], dtype=torch.float64)
    pos = (c[:, None, :] + (off[None] - 0.5) * l[:, None, :]).reshape(-1, 3).numpy()
    flat = key.reshape(-1).numpy()
    # one position per grid point, and distinct grid points have distinct positions
    first = np.full(M, -1)
    first[flat[::-1]] = np.arange(len(flat))[::-1]
    assert np.array_equal(pos, pos[first[flat]])
    assert len(np.unique(pos[first], axis=0)) == M
