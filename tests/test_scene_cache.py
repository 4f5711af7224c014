"""The scene cache: a cached scene equals a rebuilt one, entries go to the
configured private directory, and an unreadable entry is rebuilt."""
import os
import stat

import numpy as np

from sv_raster_b200 import synthetic


def test_cached_scene_equals_rebuilt(tmp_path, monkeypatch):
    d = tmp_path / "scenes"
    monkeypatch.setenv("SVR_SCENE_CACHE", str(d))
    a = synthetic.cached_config_scene("c1", n_voxels=2000)
    assert stat.S_IMODE(os.stat(d).st_mode) == 0o700
    files = os.listdir(d)
    name = f"c1_0_2000_{synthetic.generator_digest()}.pkl"
    assert files == [name]
    b = synthetic.cached_config_scene("c1", n_voxels=2000)  # from the cache
    c = synthetic.config_scene("c1", n_voxels=2000)          # rebuilt
    for x in (a, b):
        for f in ("octpath", "octlevel", "centers", "lengths", "geos", "sh0", "shs"):
            assert np.array_equal(getattr(x, f), getattr(c, f))
        assert [cam.width for cam in x.cameras] == [cam.width for cam in c.cameras]
    # a truncated entry is rebuilt, not trusted
    (d / name).write_bytes(b"\x80\x04truncated")
    e = synthetic.cached_config_scene("c1", n_voxels=2000)
    assert np.array_equal(e.centers, c.centers)


def test_every_configuration_builds_small():
    """Each benchmark configuration's generator runs (scaled down): voxels in
    the unit cube without overlapping cells, and its own camera set."""
    for name, n_cams in (("c1", 3), ("c2", 1), ("c3", 16), ("c4", 8), ("c5", 32)):
        sc = synthetic.config_scene(name, n_voxels=3000)
        assert 0 < sc.n_voxels <= 3000 and len(sc.cameras) == n_cams
        assert np.all(np.abs(sc.centers) + sc.lengths.reshape(-1, 1) / 2 <= 0.5 + 1e-6)
        assert len(np.unique(sc.octpath * 32 + sc.octlevel)) == sc.n_voxels
