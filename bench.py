"""Benchmark of the sparse-voxel rasterizer hot path on synthetic scenes.

Default workload (N=1): 8M voxels (levels 8-14, surfaces + background shell),
8 views at 1920x1080, SH degree 3.  One step = every view rendered forward and
back-propagated (projection, binning, compositing, SH, recompute backward).

  metric  fwd+bwd ms/view   (lower is better; `value` = device time per view,
                             all ranks' views / max-over-ranks time)
  e2e     the same metric through the public Python API with host buffers:
          targets and cameras copied host->device every step, loss read back.

Modes: --mode batched (one launch per stage over all views, bf16 storage of
densities / SH) or --mode plain (one view per call, fp32, the reference's
call pattern).  --impl reference times the CPU restatement of the same path
(oracle/, all host threads) on a bounded sample of the same workload.

After the timed regions, a comparator leg (batched mode, N=1) times the plain
fp32 path and the reference backend (oracle/_ref, its own per-view calls) on
the same GPU and cameras, and reports the batched and plain images' and
gradients' errors against the FP64 oracle on sampled tiles (`comparators`,
`accuracy`); --no-compare skips it.

Multi-GPU (torchrun): views are sharded, each rank renders its own views of
the shared scene; no collective in the timed data path (weak scaling).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c4", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--mode", default="batched", choices=["plain", "batched"])
    ap.add_argument("--voxels", type=int, default=None, help="override the voxel count (smaller profiles)")
    ap.add_argument("--views", type=int, default=None, help="use only the first N views")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg (profiling runs)")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the comparator leg (plain fp32 path, reference backend, FP64-oracle accuracy)")
    ap.add_argument("--no-tune", action="store_true",
                    help="batched mode: default launch parameters instead of the autotuner's choice")
    ap.add_argument("--tile", default=None,
                    help="batched mode: fixed compositing tile 'TS', 'TS,SB' or 'TS,SB,SB_backward' (8,64 | "
                         "16,128|256|512 | 32,256; the backward's staging depth apart); no autotuning")
    ap.add_argument("--bwd-walk", default=None, choices=["warp", "pair"],
                    help="batched mode with --tile: the backward with one or two pixels per thread")
    ap.add_argument("--exact", action="store_true",
                    help="batched mode: the exact compositing arithmetic (bit-identical to the plain path) instead "
                         "of the default fast form")
    ap.add_argument("--train", action="store_true",
                    help="training-step workload (fwd + bwd + fused Adam, graph-captured) vs the plain fp32 form")
    ap.add_argument("--plain-steps", type=int, default=10, help="steps of the plain form in --train mode")
    ap.add_argument("--grid", action="store_true",
                    help="--train: densities as grid points (vox_key [P,8] into a deduplicated corner grid), the "
                         "reference's training parametrisation")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def l2_note(sc, mode):
    """Whether the step's inputs exceed the 126 MB L2 (no flush between steps
    is needed then): the voxel arrays in their storage dtype plus the step's
    per-view images."""
    P = sc.n_voxels
    elem = 4 if mode == "plain" else 2
    vox = P * (8 + 12 + 4) + P * (8 + 3 + 45) * elem
    pix = sum(c.width * c.height for c in sc.cameras) * 4 * 4  # colour + T, and their gradients
    mb = (vox + pix) / 1e6
    if mb > 126:
        return f"inputs larger than L2 ({mb:.0f} MB of voxel arrays and images > 126 MB)"
    return f"inputs fit in L2 ({mb:.0f} MB of voxel arrays and images), L2 not flushed between steps"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def scene_for(args, rank, world):
    from sv_raster_b200 import synthetic
    sc = synthetic.cached_config_scene(args.config, n_voxels=args.voxels)
    from sv_raster_b200.workload import rank_cameras
    cams = sc.cameras[: args.views] if args.views else sc.cameras
    sc.cameras = rank_cameras(cams, rank, world, config=args.config)  # weak scaling: each rank its own views
    trng = np.random.default_rng(1234 + rank)
    sc.targets = [trng.uniform(0, 1, size=(3, c.height, c.width)).astype(np.float32) for c in sc.cameras]
    return sc


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)

    from sv_raster_b200 import workload
    sc = scene_for(args, rank, world)
    if args.train:
        rc = run_train(args, sc, dev, world, rank)
        if world > 1:
            dist.destroy_process_group()
        return rc
    if args.mode == "plain":
        wl = workload.PlainWorkload(sc, dev)
    else:
        tile = None
        if args.tile:
            parts = [int(x) for x in args.tile.split(",")]
            tile = (parts[0], parts[1] if len(parts) > 1 else (64 if parts[0] == 8 else 256)) + tuple(parts[2:3])
        wl = workload.BatchedWorkload(sc, dev, tune=not (args.no_tune or tile), tile=tile, exact=args.exact,
                                      bwd_walk=args.bwd_walk if tile else None)
    n_views = len(sc.cameras)

    for _ in range(args.warmup):
        wl.step()
    torch.cuda.synchronize()

    # Timed region: K steps bracketed by barrier + sync, CUDA events on the
    # launch stream.  Batched mode replays the captured step graph (its
    # production form); plain mode runs the reference's per-view calls.
    stream = torch.cuda.current_stream(dev)
    sampler = ClockSampler(dev.index if dev.index is not None else 0)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        wl.step()
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    if hasattr(wl, "check_errors"):
        wl.check_errors()  # capacity / consistency flags of the batched step
    ms_total = workload.max_over_ranks(ev0.elapsed_time(ev1), device=dev)
    ms_per_step = ms_total / args.steps
    views_all = n_views * world
    value = ms_total / (args.steps * views_all)  # device ms per view over the whole job

    # Per-kernel durations (roofline): the same K steps again, launched eagerly
    # with CUDA events around every stage on the launch stream.
    wl.reset_kernel_timers()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        wl.step()
    t1.record(stream)
    torch.cuda.synchronize()
    eager_ms = workload.max_over_ranks(t0.elapsed_time(t1), device=dev) / args.steps
    kstats = wl.kernel_stats()
    wl.timers = {}

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = wl.e2e(args.steps, args.warmup)
        e2e["ms_total"] = workload.max_over_ranks(e2e["ms_total"], device=dev)
    r = getattr(wl, "raster", None)
    # committed-capture lookup keys of the compositing kernels: tile size and staging depth
    tile_keys = ({"render_fwd": f"{r.tile_size},{r.staging}",
                  "render_bwd": f"{r.tile_size},{r.staging_bwd or r.staging}"} if r is not None else
                 {"render_fwd": "16,256", "render_bwd": "16,256"})
    inst_per_view = wl.instances_per_view()
    launches = wl.launches_per_step()
    tuned = getattr(wl, "tuned", None)
    r = None

    # Comparator leg (rank 0, N=1; after every timing of this path): the plain
    # fp32 per-view path on the same scene and cameras, the reference backend's
    # own per-view call sequence on the same GPU, and image / gradient errors
    # against the FP64 oracle on sampled tiles of view 0.
    comparators = None
    if rank == 0 and world == 1 and not args.no_compare and args.mode == "batched":
        kstats_keep = kstats
        del wl
        torch.cuda.empty_cache()
        comparators = comparator_leg(args, sc, dev, value)
        kstats = kstats_keep

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(sc, budget_s=15.0)

    if rank == 0:
        peak, peak_kind = load_peaks()
        dom = kstats["dominant"]
        achieved = dom["bytes"] / (dom["ms"] * 1e-3) / 1e9 if dom["ms"] > 0 else 0.0
        # measured DRAM bytes per launch: committed ncu capture of the same
        # kernel on a smaller case, scaled by instances per launch
        traffic = None
        issue = None
        tf = os.path.join(ROOT, "profiles", "render_traffic.json")
        if os.path.exists(tf) and dom["name"] in ("render_fwd", "render_bwd"):
            t = json.load(open(tf))["tiles"].get(tile_keys[dom["name"]])
            if t is not None:
                inst = inst_per_view * (n_views if args.mode == "batched" else 1)
                traffic = round(t[dom["name"]]["dram_bytes"] / t["instances_per_launch"] * inst)
                # the compositing kernels are bounded by instruction issue, not HBM
                ipc = t[dom["name"]].get("ipc")
                if ipc:
                    issue = {"ipc": ipc, "peak_ipc": 4.0, "frac": round(ipc / 4.0, 3),
                             "source": "profiles/render_traffic.json (committed ncu capture, small case)"}
        line = {
            "metric": "fwd+bwd ms/view", "value": round(value, 4), "unit": "ms/view", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "storage_dtype": "f32" if args.mode == "plain" else "bf16", "data": "synthetic",
            "config": {"workload": f"{args.config}: {sc.n_voxels} voxels, {n_views} views/rank "
                                   f"{sc.cameras[0].width}x{sc.cameras[0].height}, SH3, fwd+recompute bwd",
                       "mode": args.mode, "l2": l2_note(sc, args.mode),
                       "arithmetic": ("exact" if args.exact or args.mode == "plain" else "fast"),
                       "instances_per_view": inst_per_view,
                       "scene_file": os.path.basename(scene_file(args))},
            "autotuned": tuned,
            "render_fps": round(1000.0 / kstats["fwd_ms_per_view"], 2) if kstats.get("fwd_ms_per_view") else None,
            "rays_per_s": round(sum(c.width * c.height for c in sc.cameras) * world / (ms_total / args.steps * 1e-3),
                                1),
            "gpu_launches": launches * args.steps,
            "timed_form": "cuda-graph replay" if args.mode == "batched" else "eager per-view calls",
            "eager_instrumented_ms_per_step": round(eager_ms, 4),
            "roofline": {"bound": "hbm", "kernel": dom["name"], "achieved": round(achieved, 2),
                         "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": dom["bytes_per_launch"],
                         "ms_per_launch": round(dom["ms_per_launch"], 4), "issue": issue},
            "kernels": kstats["table"],
            "clocks": clocks,
        }
        if e2e is not None:
            line["e2e"] = {"value": round(e2e["ms_total"] / (args.steps * views_all), 4), "unit": "ms/view",
                           "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"]}
        if comparators is not None:
            line["comparators"] = comparators.pop("timing")
            line["accuracy"] = comparators.pop("accuracy")
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_train(args, sc, dev, world, rank):
    """Training-step comparison: batched bf16-storage step (one CUDA graph,
    fused Adam with the step count on the device) against the plain fp32
    reference-pattern step, from the same initial parameters."""
    import torch
    from sv_raster_b200 import workload
    torch.cuda.set_device(dev)
    torch.zeros(1, device=dev)
    torch.cuda.reset_peak_memory_stats()
    exchange = workload.GradientExchange() if world > 1 else None
    grid = None
    if args.grid:
        from sv_raster_b200 import synthetic
        grid = synthetic.grid_params(sc, dev)
    wl = workload.BatchedTrainWorkload(sc, dev, exchange=exchange, grid=grid)
    wl.capture()
    peak_setup = torch.cuda.max_memory_allocated()  # includes the autotuner's trial plans
    torch.cuda.reset_peak_memory_stats()
    ms_b, loss_b = wl.run(args.steps)
    ms_b = workload.max_over_ranks(ms_b, device=dev)
    peak_b = torch.cuda.max_memory_allocated()
    wl.release()
    del wl
    torch.cuda.empty_cache()
    ms_p = loss_p = peak_p = dev_rel = None
    if world == 1:  # the plain per-view form is the single-GPU comparator
        torch.cuda.reset_peak_memory_stats()
        wp = workload.PlainTrainWorkload(sc, dev, grid=grid)
        ms_p, loss_p = wp.run(args.plain_steps)
        peak_p = torch.cuda.max_memory_allocated()
        n = min(len(loss_b), len(loss_p))
        dev_rel = max(abs(a - b) / abs(b) for a, b in zip(loss_b[:n], loss_p[:n]))
    if rank == 0:
        print(json.dumps({
            "metric": "training ms/step", "value": round(ms_b, 3), "unit": "ms/step", "higher_is_better": False,
            "n_gpus": world, "steps": args.steps, "data": "synthetic", "dtype": "f32", "storage_dtype": "bf16",
            "config": {"workload": f"{args.config}: {sc.n_voxels} voxels, {len(sc.cameras)} views per step "
                                   f"({sc.cameras[0].width}x{sc.cameras[0].height} ... mixed), fwd + recompute bwd "
                                   f"+ fused Adam, one CUDA graph per step",
                       "densities": (f"{grid[1].shape[0]} grid points gathered per step (vox_key [P,8])"
                                     if grid is not None else "per-voxel corners [P,8]")},
            "scaling": "weak",
            "exchange": "sum all-reduce of the flat gradient buffer per step (NCCL)" if world > 1 else None,
            "plain_fp32": None if ms_p is None else {"ms_per_step": round(ms_p, 3), "steps": args.plain_steps,
                                                     "untimed_first_steps": min(2, max(args.plain_steps - 1, 0)),
                                                     "peak_hbm_gb": round(peak_p / 1e9, 2)},
            "speedup_vs_plain": None if ms_p is None else round(ms_p / ms_b, 3),
            "peak_hbm_gb": round(peak_b / 1e9, 2),
            "peak_hbm_gb_incl_setup": round(peak_setup / 1e9, 2),
            "loss_batched_bf16": [round(x, 6) for x in loss_b],
            "loss_plain_fp32": None if loss_p is None else [round(x, 6) for x in loss_p],
            "loss_max_rel_dev_common_steps": None if dev_rel is None else round(dev_rel, 6)}), flush=True)
    return 0


def scene_file(args):
    """Cache file the scene of this run was loaded from (or written to)."""
    from sv_raster_b200 import synthetic
    return synthetic.cached_scene_path(args.config, n_voxels=args.voxels)


def _timed_steps(step, steps, warmup, dev):
    """Device ms of `steps` calls of `step` after `warmup` untimed ones (CUDA
    events on the current stream) and the clocks sampled meanwhile."""
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index if dev.index is not None else 0)
    sampler.start()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        step()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), sampler.stop()


def comparator_leg(args, sc, dev, batched_ms_per_view):
    """The north-star comparators on the same GPU, scene and cameras, after the
    batched path's timing: (1) this repository's plain fp32 path in the
    reference's per-view call pattern; (2) the reference backend itself
    (compiled from its sources into oracle/_ref) through its own per-view
    call sequence; (3) errors of the batched bf16-storage and plain fp32 images
    and gradients against the FP64 oracle on a seeded sample of tiles of view
    0.  The oracle and the reference module are used here as comparators and
    checker only, never inside the timed path."""
    import torch
    from sv_raster_b200 import workload
    n_views = len(sc.cameras)
    timing = {}
    wp = workload.PlainWorkload(sc, dev)
    ms, clk = _timed_steps(wp.step, args.steps, args.warmup, dev)
    timing["plain_fp32"] = {"ms_per_view": round(ms / (args.steps * n_views), 4), "clocks": clk,
                            "form": "this repository's plain path, fp32, one view per call with the reference's "
                                    "host syncs (instance count, visible-index read)"}
    del wp
    torch.cuda.empty_cache()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        from time_reference_gpu import ReferenceSteps
        rs = ReferenceSteps(sc, sc.cameras, dev)
    except (ImportError, OSError) as e:
        timing["reference_gpu"] = {"unavailable": f"reference backend module not loadable: {e}"}
        rs = None
    if rs is not None:
        ms, clk = _timed_steps(rs.step, args.steps, args.warmup, dev)
        timing["reference_gpu"] = {"ms_per_view": round(ms / (args.steps * n_views), 4), "clocks": clk,
                                   "form": "reference CUDA backend (backends/cuda, compiled from its sources), its "
                                           "per-view call sequence: preprocess, visible-index sync, SH, forward "
                                           "(instance-count sync), L2-loss gradient, backward, SH backward; fp32"}
        del rs
        torch.cuda.empty_cache()
    for k in ("plain_fp32", "reference_gpu"):
        v = timing[k].get("ms_per_view")
        if v:
            timing[f"batched_over_{k}"] = round(v / batched_ms_per_view, 3)
    import accuracy
    cam = sc.cameras[0]
    t0 = time.perf_counter()
    acc = accuracy.measure(sc, cam, sc.targets[0])
    acc["view"] = f"view 0 ({cam.width}x{cam.height}), {acc['tiles']} of " \
                  f"{((cam.width + 15) // 16) * ((cam.height + 15) // 16)} 16x16 tiles (seeded runs of 16)"
    acc["seconds"] = round(time.perf_counter() - t0, 1)
    return {"timing": timing, "accuracy": acc}


def cpu_baseline(sc, budget_s=15.0, view=0, seed=0):
    """The CPU oracle (fp32 mimic, all host threads) on a bounded sample of one
    view: its full SH, projection and binning, then forward + backward of
    seeded runs of 128 tiles spread over the image until the budget is spent;
    reported as ms/view = setup + mean time per sampled tile x tile count.
    (Each oracle call allocates full-view images and per-voxel gradients, so
    runs are long enough for the compositing to dominate the sample.)"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cam = sc.cameras[view % len(sc.cameras)]
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    t0 = time.perf_counter()
    ndup, bbox, quad = O.preprocess(cam, sc.centers, sc.lengths)
    vis = np.nonzero(ndup)[0]
    rgbs = O.sh_fwd(3, vis, sc.centers, cam.position, sc.sh0, sc.shs)
    keys, vals, ranges = O.binning(cam, sc.octpath, ndup, bbox, quad)
    t_setup = time.perf_counter() - t0
    gx, gy = (cam.width + 15) // 16, (cam.height + 15) // 16
    T = gx * gy
    run = 128
    order = np.random.default_rng(seed + view).permutation(max(1, -(-T // run)))
    spent, done = 0.0, 0
    for slot in order:
        lo, hi = int(slot) * run, min(T, int(slot) * run + run)
        t1 = time.perf_counter()
        out = O.render_fwd(cam, ranges, vals, bbox, sc.centers, sc.lengths, sc.geos, rgbs, tiles=(lo, hi))
        dC = np.full_like(out["color"], 1e-3)
        O.render_bwd(cam, ranges, out["tile_last"], vals, bbox, sc.centers, sc.lengths, sc.geos, rgbs,
                     out["n_contrib"], out["T"], dC, np.zeros_like(out["T"], dtype=np.float32), tiles=(lo, hi))
        spent += time.perf_counter() - t1
        done += hi - lo
        if spent + t_setup >= budget_s:
            break
    ms_view = (spent / max(done, 1) * T + t_setup) * 1e3
    return {"value": round(ms_view, 2), "unit": "ms/view", "cores": cores, "kind": "port",
            "sample": f"view {view % len(sc.cameras)}: full SH + projection + binning ({len(vals)} instances, "
                      f"{t_setup:.1f} s) + fwd/bwd of {done} of {T} 16x16 tiles in seeded runs of {run} over the "
                      f"image ({spent:.1f} s), per-tile mean x tile count"}


def run_reference(args):
    """Reference arm: the CPU restatement of the reference path (oracle port,
    all host threads) on a bounded sample of the same workload."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sc = scene_for(args, 0, 1)
    per_step = min(30.0, max(5.0, 60.0 / max(1, args.steps)))
    if args.warmup > 0:
        cpu_baseline(sc, budget_s=1.0)
    vals = [cpu_baseline(sc, budget_s=per_step, view=k) for k in range(max(1, args.steps))]
    v = float(np.median([x["value"] for x in vals]))
    line = {"metric": "fwd+bwd ms/view", "value": round(v, 2), "unit": "ms/view", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"{args.config}: {sc.n_voxels} voxels, {len(sc.cameras)} views "
                                   f"{sc.cameras[0].width}x{sc.cameras[0].height}", "mode": "cpu"},
            "cpu_baseline": {"value": round(v, 2), "unit": "ms/view", "cores": vals[0]["cores"], "kind": "port",
                             "sample": f"median of {len(vals)} per-step samples, step k on view k mod "
                                       f"{len(sc.cameras)}; step 0: {vals[0]['sample']}"},
            "e2e": {"value": round(v, 2), "unit": "ms/view", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
