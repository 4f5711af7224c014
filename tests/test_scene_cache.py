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
