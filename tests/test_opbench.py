"""The operator benchmark: its grid builder (CPU; corner indices of octree
voxels into a deduplicated grid address one point per distinct corner
position) and one small end-to-end run (GPU)."""
import numpy as np
import pytest
import torch

from sv_raster_b200 import synthetic
from sv_raster_b200.synthetic import grid_keys


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


@pytest.mark.gpu
def test_opbench_runs_on_a_small_scene(tmp_path):
    """The operator benchmark end to end on a 20k-voxel scene: every operator
    timed, no error."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "opbench.py"), "--voxels", "20000", "--reps", "1",
                          "--warmup", "1"], cwd=root, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert set(res["ops"]) >= {"gather_geo", "gather_geo_bw", "gather_feat", "gather_feat_bw", "tv_bw",
                               "tv_bw_sparse", "render_fwd_plain", "render_bwd_depth_normal_dist"}
    assert all(v["ms"] > 0 for v in res["ops"].values())
