"""CPU tests of the autotuner's search and cache logic with a fake
rasterizer and a fake timer (the GPU test in test_gpu_batched.py runs it on
the real kernels)."""
import torch

from sv_raster_b200 import autotune


class FakeRaster:
    def __init__(self):
        self.dev = torch.device("cpu")
        self.P = 1000
        self.sizes = [(32, 48), (16, 16)]
        self.n_samp = 1
        self.n_pixels = 32 * 48 + 16 * 16
        self.tile_size, self.staging = 16, 256
        self.sort_buckets = (512, 4096)
        self.schedule = (3, 0, 0)
        self.fits = 0

    def set_tile_size(self, t, s=None):
        self.tile_size, self.staging = t, s
        self.staging_bwd = None

    def set_staging(self, s):
        if s not in ((32, 64, 128) if self.tile_size == 8 else (128, 256, 512)):
            raise RuntimeError("staging depth not supported by this tile size")
        self.staging, self.staging_bwd = s, None

    def set_sort_buckets(self, a, b):
        self.sort_buckets = (a, b)

    def set_reduction(self, k):
        self.atomic_lanes = k

    def set_binning(self, b):
        self.binning = b

    def set_pixels_per_thread(self, n):
        self.pixels_per_thread = n

    def set_backward_pixels_per_thread(self, n=None):
        self.pixels_per_thread_bwd = n

    def set_backward_staging(self, n=None):
        if n is not None and n not in ((32, 64, 128) if self.tile_size == 8 else (128, 256, 512)):
            raise RuntimeError("staging depth not supported by this tile size")
        self.staging_bwd = n

    def set_schedule(self, fwd_ordered=True, bwd_ordered=True, fwd_ctas_per_sm=0, bwd_ctas_per_sm=0):
        self.schedule = (int(fwd_ordered) | (int(bwd_ordered) << 1), fwd_ctas_per_sm, bwd_ctas_per_sm)

    def fit_capacity(self, *a):
        self.fits += 1
        return 1

    def prepare(self, *a):
        pass

    def render(self, geos, color=None, T=None):
        return torch.zeros(3 * self.n_pixels), torch.zeros(self.n_pixels)

    def backward(self, *a, **k):
        return a[-1] if len(a) > 6 else None


def test_tuner_picks_fastest_per_stage_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("SVR_AUTOTUNE_CACHE", str(tmp_path / "c.json"))
    r = FakeRaster()

    # cost model: tile 8 fastest, sort (256, 4096) fastest, fwd unordered with cap 4... etc.
    def timer(fn, reps, warmup):
        fn()
        t = 10.0
        t -= {8: 3.0, 32: 1.0}.get(r.tile_size, 0.0)
        t -= 2.0 if r.sort_buckets == (256, 4096) else 0.0
        t -= 1.5 if (r.schedule[0] & 1) == 0 else 0.0
        t -= 0.5 * (r.schedule[2] == 3)
        t -= 0.25 * (getattr(r, "atomic_lanes", 1) == 4)
        t -= 0.125 * (getattr(r, "binning", 1) == 0)
        t -= 0.0625 * (getattr(r, "pixels_per_thread", 1) == 2)
        t -= 0.03125 * (getattr(r, "staging_bwd", None) == 32)
        t -= 0.015625 * (r.staging == 128 and getattr(r, "staging_bwd", None) == 32)
        t -= 0.0078125 * (getattr(r, "pixels_per_thread_bwd", None) == 1)
        return t

    geos = torch.zeros(r.P, 8)
    sh0, shs = torch.zeros(r.P, 3), torch.zeros(r.P, 15, 3)
    space = dict(autotune.DEFAULT_SPACE, bwd=[(True, 0), (False, 0), (True, 3), (True, 2)])
    res = autotune.tune_batched(r, geos, sh0, shs, 3, space=space, timer=timer)
    assert not res["cached"]
    assert res["choice"]["tile"] == (8, 64)
    assert res["choice"]["sort"] == (256, 4096)
    assert res["choice"]["fwd"] == (False, 0)
    assert res["choice"]["bwd"] == (True, 3)
    # the chosen parameters are left applied
    assert (r.tile_size, r.staging, r.sort_buckets) == (8, 128, (256, 4096))  # forward depth re-tuned
    assert r.schedule == (2, 0, 3)
    assert res["choice"]["reduce"] == 4 and r.atomic_lanes == 4
    assert res["choice"]["bin"] == 0 and r.binning == 0
    assert res["choice"]["ppt"] == 2 and r.pixels_per_thread == 2
    assert res["choice"]["bppt"] == 1 and r.pixels_per_thread_bwd == 1  # the backward's own
    assert res["choice"]["bstage"] == 32 and r.staging_bwd == 32
    assert [c for c, _ in res["timings"]["bstage"]] == [0, 32, 64, 128]  # 256 needs 16x16 tiles
    # the forward's own depth, re-tuned with the backward's kept
    assert res["choice"]["fstage"] == 128 and r.staging == 128 and r.staging_bwd == 32
    assert set(res["timings"]) == {"tile", "ppt", "bppt", "bstage", "fstage", "bin", "sort", "fwd", "bwd", "reduce"}
    # second call: served from the cache, applied, no timing
    r2 = FakeRaster()
    res2 = autotune.tune_batched(r2, geos, sh0, shs, 3, timer=lambda *a: 1 / 0)
    assert res2["cached"] and res2["choice"] == res["choice"]
    assert (r2.tile_size, r2.sort_buckets, r2.schedule) == (8, (256, 4096), (2, 0, 3))
    assert r2.fits == 1


def test_tuner_restricted_space_and_no_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("SVR_AUTOTUNE_CACHE", str(tmp_path / "c.json"))
    r = FakeRaster()
    space = {"fwd": [(True, 0), (True, 4)]}
    res = autotune.tune_batched(r, torch.zeros(1), torch.zeros(1, 3), torch.zeros(1, 15, 3), 3, space=space,
                                cache=False, timer=lambda fn, reps, w: 5.0 - r.schedule[1])
    assert res["choice"]["fwd"] == (True, 4)
    assert set(res["timings"]) == {"fwd"}
    assert not (tmp_path / "c.json").exists()
