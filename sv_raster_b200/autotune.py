"""Autotuner for the batched rasterizer's launch parameters.

The parameters it chooses change only how the work is scheduled, never the
results (images and contributor counts are bit-identical across choices;
gradients agree up to the order of floating-point additions):

* ``fwd`` / ``bwd`` -- compositing schedule of the persistent forward and
  backward launches: tiles largest first or in tile order
  (``BatchedRasterizer.set_schedule``; its cap on resident CTAs per SM can be
  searched too by listing ``(ordered, cap)`` pairs, but full occupancy won on
  every scene measured, so the default space leaves it out).
* ``bin`` -- how instances are grouped by tile before the per-tile sort:
  counting sort with atomics (1) or radix passes over the tile bits (0)
  (``BatchedRasterizer.set_binning``).
* ``sort`` -- segment-size buckets of the per-tile segment sort: the largest
  segment sorted by one small CTA and the chunk length of the chunked sort
  (``BatchedRasterizer.set_sort_buckets``).
* ``reduce`` -- backward gradient reduction threshold: records touched by at
  most this many lanes of a warp add their gradients with shared-memory
  atomics instead of a warp reduce-scatter (``set_reduction``).
* ``bstage`` -- the backward's own staging depth (0: the forward's), tuned
  with the backward after the tile (``set_backward_staging``): the backward
  holds more per-record state in shared memory, so a shallower staging round
  can keep more CTAs resident.  Depths the tile size does not support are
  skipped.
* ``fstage`` -- the forward's staging depth once the backward's is set apart
  (0: the tile's own), timed with the forward alone; the tile stage times
  both kernels with one depth, and the two kernels prefer different ones
  (c4: forward 64, backward 32 records).
* ``ppt`` -- pixels per compositing thread, 1 or 2 (two pixels of an 8x8
  warp block share each record's loads and, in the backward, its warp
  reduction; ``BatchedRasterizer.set_pixels_per_thread``), timed with the
  forward after the tile.
* ``bppt`` -- the backward's own pixels per thread (0: as ``ppt``), timed
  with the backward: the forward walks each pixel's own records, which two
  pixels per thread cannot, while the backward's warp reduction favours two
  (``set_backward_pixels_per_thread``).
* ``tile`` -- compositing tile size of the batched path (8, 16 or 32 pixels)
  with the voxel-staging depth (records staged into shared memory per round)
  (``BatchedRasterizer.set_tile_size``; the tile size changes the binning, so
  it is tuned with the full step).

Each stage is timed on the caller's own scene and cameras with CUDA events
(median of ``reps`` launches after warm-up), one stage at a time, and the
fastest candidate is kept.  Results are cached in a JSON file keyed by the
GPU, the scene size, the camera sizes and the storage dtypes
(``SVR_AUTOTUNE_CACHE`` overrides the path; ``cache=False`` skips it).
"""
import json
import os

import torch

DEFAULT_SPACE = {
    "tile": [(16, 256), (8, 64), (8, 32), (8, 128), (16, 128), (16, 512), (32, 256)],
    "bin": [1, 0],
    "sort": [(512, 4096), (256, 4096), (1024, 4096), (512, 2048)],
    "fwd": [(True, 0), (False, 0)],
    "bwd": [(True, 0), (False, 0)],
    "reduce": [1, 2, 4, 8],
    "ppt": [1, 2],
    "bppt": [0, 1, 2],
    "bstage": [0, 32, 64, 128, 256],
    "fstage": [0, 32, 64, 128, 256, 512],
}


def cache_path():
    return os.environ.get("SVR_AUTOTUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "sv_raster_b200", "autotune.json")


def _load_cache(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(path, data):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


# Bumped whenever the search space or the kernels behind it change, so that
# choices cached by an older build are measured again rather than reused.
CACHE_SCHEMA = 7


def cache_key(raster, geos, sh0):
    dev = raster.dev
    name = torch.cuda.get_device_name(dev) if dev.type == "cuda" else "cpu"
    sizes = ",".join(f"{w}x{h}" for h, w in raster.sizes)
    return (f"v{CACHE_SCHEMA}|{name}|P={raster.P}|views={sizes}|ns={raster.n_samp}|geo={geos.dtype}"
            f"|sh={sh0.dtype}|arith={'exact' if getattr(raster, 'exact', False) else 'fast'}")


def time_ms(fn, reps=5, warmup=2, stream=None):
    """Median device time of fn() in ms (CUDA events on the current stream)."""
    st = stream or torch.cuda.current_stream()
    for _ in range(warmup):
        fn()
    times = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    times.sort()
    return times[len(times) // 2]


def apply(raster, choice):
    """Apply a tuned choice dict (keys of DEFAULT_SPACE) to a rasterizer."""
    if "tile" in choice:
        ts, sb = choice["tile"]
        raster.set_tile_size(int(ts), int(sb))
    if "bin" in choice:
        raster.set_binning(int(choice["bin"]))
    if "sort" in choice:
        raster.set_sort_buckets(*[int(x) for x in choice["sort"]])
    if "reduce" in choice:
        raster.set_reduction(int(choice["reduce"]))
    if "ppt" in choice:
        raster.set_pixels_per_thread(int(choice["ppt"]))
    if "bppt" in choice:
        raster.set_backward_pixels_per_thread(int(choice["bppt"]) or None)
    if int(choice.get("fstage", 0)):
        raster.set_staging(int(choice["fstage"]))  # (resets the backward's; set again below)
    if "bstage" in choice:
        raster.set_backward_staging(int(choice["bstage"]) or None)
    f = choice.get("fwd", (True, 0))
    b = choice.get("bwd", (True, 0))
    raster.set_schedule(fwd_ordered=bool(f[0]), bwd_ordered=bool(b[0]), fwd_ctas_per_sm=int(f[1]),
                        bwd_ctas_per_sm=int(b[1]))


def tune_batched(raster, geos, sh0, shs, sh_degree=3, space=None, reps=5, warmup=2, cache=True, timer=time_ms):
    """Choose the batched rasterizer's launch parameters for this scene.

    Returns ``dict(choice=..., timings=..., cached=bool)`` and leaves the
    choice applied to ``raster``.  ``timer(fn, reps, warmup)`` times a stage
    (replaceable for tests).  Stages are tuned in order: tile size (full
    step), binning and sort buckets (prepare), forward schedule (render), backward
    schedule (backward), each with the previous choices applied.
    """
    space = dict(DEFAULT_SPACE if space is None else space)
    key = cache_key(raster, geos, sh0)
    path = cache_path()
    if cache:
        hit = _load_cache(path).get(key)
        if hit is not None:
            choice = {k: (tuple(v) if isinstance(v, list) else v) for k, v in hit["choice"].items()}
            apply(raster, choice)
            raster.fit_capacity(sh0, shs, sh_degree)
            return dict(choice=choice, timings=hit.get("timings", {}), cached=True)

    M = 1 + shs.shape[1]
    choice = {name: cands[0] for name, cands in DEFAULT_SPACE.items()}
    timings = {}
    gen = torch.Generator(device=raster.dev)
    gen.manual_seed(0)
    state = {}

    def upstream():
        # a fixed, seeded upstream gradient of the images (values do not matter for timing)
        if "dC" not in state or state["dC"].numel() != 3 * raster.n_pixels:
            state["dC"] = torch.rand(3 * raster.n_pixels, device=raster.dev, generator=gen) * 1e-6
            state["dT"] = torch.zeros(raster.n_pixels, device=raster.dev)
        return state["dC"], state["dT"]

    def step():
        raster.prepare(sh0, shs, sh_degree)
        render()
        backward()

    def prepare():
        raster.prepare(sh0, shs, sh_degree)

    def render():
        state["out"] = raster.render(geos, *state.get("out", (None, None)))

    def backward():
        dC, dT = upstream()
        state["grads"] = raster.backward(geos, state["out"][1], dC, dT, sh_degree, M, state.get("grads"))

    stages = [("tile", step), ("ppt", render), ("bppt", backward), ("bstage", backward), ("fstage", render), ("bin", prepare),
              ("sort", prepare), ("fwd", render), ("bwd", backward), ("reduce", backward)]
    for name, fn in stages:
        cands = space.get(name)
        if not cands:
            continue
        res = []
        for cand in cands:
            try:
                apply(raster, dict(choice, **{name: cand}))
            except RuntimeError:  # a value this tile configuration does not support
                continue
            if name == "tile":
                raster.fit_capacity(sh0, shs, sh_degree)
            if name in ("ppt", "bppt", "fwd", "bwd", "reduce", "bstage", "fstage"):
                raster.prepare(sh0, shs, sh_degree)
                render()
            t = timer(fn, reps, warmup)
            res.append((t, cand))
        timings[name] = [[c if not isinstance(c, tuple) else list(c), round(t, 4)] for t, c in res]
        choice[name] = min(res, key=lambda x: x[0])[1]
        if name in ("bstage", "fstage") and not choice[name]:
            choice[name] = raster.staging  # "as the tile's" made concrete: later stages may change it
        if name == "bppt" and not choice[name]:
            choice[name] = choice["ppt"]
        apply(raster, choice)
        if name == "tile":
            raster.fit_capacity(sh0, shs, sh_degree)
    if cache:
        data = _load_cache(path)
        data[key] = dict(choice={k: (list(v) if isinstance(v, tuple) else v) for k, v in choice.items()},
                         timings=timings)
        _store_cache(path, data)
    return dict(choice=choice, timings=timings, cached=False)
