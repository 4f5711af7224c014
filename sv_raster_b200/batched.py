"""Multi-view batched rasterization: many cameras of uneven resolution over
one shared voxel set, one launch per stage, no host round trip, CUDA-graph
capturable.  Densities and SH coefficients may be stored in bf16; all
compositing, transmittance and gradient accumulation is fp32.

This has no counterpart in the reference (which renders one view per call);
per view it produces the plain path's images, contributor counts and tile
lists.
"""
import ctypes
import math

import torch

from ._native import Camera, check, lib

TILE = 16


class BatchedRasterizer:
    """A plan over fixed cameras + a workspace sized for the scene.

    ``cameras``: objects with width, height, tanfovx, tanfovy, cx, cy, near and
    device tensors ``w2c`` / ``c2w`` (4x4 fp32).  The device addresses of
    those matrices are baked into the plan; update them in place to move the
    cameras (e.g. between CUDA-graph replays).  ``max_level`` bounds the
    voxels' octree levels (shorter sort keys; checked on the device).
    ``exact`` selects the compositing arithmetic (see set_arithmetic).
    """

    def __init__(self, cameras, octree_paths, vox_centers, vox_lengths, max_level=16, n_samp_per_vox=1,
                 bg_color=0.0, capacity=None, headroom=1.25, tile_size=16, exact=False):
        self.dev = vox_centers.device
        self.cams = list(cameras)
        self.octree_paths = octree_paths.reshape(-1).contiguous()
        self.centers = vox_centers.contiguous()
        self.lengths = vox_lengths.contiguous()
        self.P = self.centers.shape[0]
        self.max_level = int(max_level)
        self.n_samp = int(n_samp_per_vox)
        self.bg = float(bg_color)
        self.headroom = headroom
        self._c_cams = (Camera * len(self.cams))()
        for i, c in enumerate(self.cams):
            if c.w2c.device != self.dev or c.c2w.device != self.dev:
                raise ValueError("camera matrices must live on the voxels' device")
            self._c_cams[i] = Camera(c.width, c.height, c.tanfovx, c.tanfovy, c.cx, c.cy, c.w2c.data_ptr(),
                                     c.c2w.data_ptr(), c.near, self.bg)
        self.sizes = [(c.height, c.width) for c in self.cams]
        self.pix_offsets = [0]
        for h, w in self.sizes:
            self.pix_offsets.append(self.pix_offsets[-1] + h * w)
        self.plan = None
        self.tile_size = int(tile_size)
        self.staging = 64 if self.tile_size == 8 else 256
        self.schedule = (3, 0, 0)
        self.sort_buckets = (512, 4096)
        self.atomic_lanes = 1
        self.binning = 1
        self.exact = bool(exact)
        self.pixels_per_thread = 1
        self.pixels_per_thread_bwd = None  # None: as pixels_per_thread
        self.culling = -1  # -1: tight bbox with the fast arithmetic, the rounded one with the exact
        self.staging_bwd = None  # None: the forward's staging depth
        self._make_plan(0 if capacity is None else int(capacity))
        self.capacity_auto = capacity is None

    # -- plan / workspace ----------------------------------------------------
    def _make_plan(self, capacity):
        L = lib()
        if self.plan is not None:
            L.svr_batch_plan_destroy(self.plan)
            self.plan = None
        plan = ctypes.c_void_p()
        nbytes = ctypes.c_size_t()
        check(L.svr_batch_plan_create(len(self.cams), self._c_cams, self.P, capacity, self.n_samp, self.max_level,
                                      self.tile_size, ctypes.byref(plan), ctypes.byref(nbytes)), "batch_plan_create")
        self.plan = plan
        self.capacity = capacity
        self.ws = torch.empty(nbytes.value, dtype=torch.uint8, device=self.dev)
        self.n_pixels = int(L.svr_batch_plan_pixels(plan))
        self.n_tiles = int(L.svr_batch_plan_tiles(plan))
        self.n_groups = int(L.svr_batch_plan_groups(plan))
        check(L.svr_batch_plan_set_schedule(plan, *self.schedule), "batch_plan_set_schedule")
        check(L.svr_batch_plan_set_sort_buckets(plan, *self.sort_buckets), "batch_plan_set_sort_buckets")
        check(L.svr_batch_plan_set_staging(plan, self.staging), "batch_plan_set_staging")
        check(L.svr_batch_plan_set_reduction(plan, self.atomic_lanes), "batch_plan_set_reduction")
        check(L.svr_batch_plan_set_binning(plan, self.binning), "batch_plan_set_binning")
        check(L.svr_batch_plan_set_arithmetic(plan, int(self.exact)), "batch_plan_set_arithmetic")
        check(L.svr_batch_plan_set_culling(plan, self.culling), "batch_plan_set_culling")
        check(L.svr_batch_plan_set_pixels_per_thread(plan, self.pixels_per_thread),
              "batch_plan_set_pixels_per_thread")
        check(L.svr_batch_plan_set_backward_pixels_per_thread(plan, self.pixels_per_thread_bwd or 0),
              "batch_plan_set_backward_pixels_per_thread")
        if self.staging_bwd is not None:
            check(L.svr_batch_plan_set_backward_staging(plan, self.staging_bwd), "batch_plan_set_backward_staging")

    def set_binning(self, binning=1):
        """How prepare groups the instances by tile before the per-tile sort:
        1 a counting sort (counts, scan, atomic scatter), 0 radix passes over
        the tile bits.  The sorted lists are the same."""
        check(lib().svr_batch_plan_set_binning(self.plan, int(binning)), "batch_plan_set_binning")
        self.binning = int(binning)

    def set_reduction(self, atomic_lanes=1):
        """Backward: records with at most ``atomic_lanes`` contributing lanes
        in a warp add their gradients with shared atomics instead of the warp
        reduce-scatter (only the order of additions changes)."""
        check(lib().svr_batch_plan_set_reduction(self.plan, int(atomic_lanes)), "batch_plan_set_reduction")
        self.atomic_lanes = int(atomic_lanes)

    def set_arithmetic(self, exact=False):
        """Compositing arithmetic: ``exact`` reproduces the plain path (and the
        reference) bit for bit; the default fast form uses the hardware
        exponential and an approximate division in the per-(pixel, voxel)
        loops (see svr_batch_plan_set_arithmetic)."""
        check(lib().svr_batch_plan_set_arithmetic(self.plan, int(bool(exact))), "batch_plan_set_arithmetic")
        self.exact = bool(exact)

    def set_culling(self, culling=-1):
        """Pixel bbox of each (view, voxel) pair: 0 the reference's rounded
        bbox (the plain path's tile lists), 1 only the pixels whose centre ray
        can meet the cube (fewer instances, same images and gradients), -1
        tight with the fast arithmetic and rounded with the exact one (see
        svr_batch_plan_set_culling).  Re-fit the capacity after switching from
        tight to rounded."""
        check(lib().svr_batch_plan_set_culling(self.plan, int(culling)), "batch_plan_set_culling")
        self.culling = int(culling)

    def set_pixels_per_thread(self, pixels=1):
        """Pixels per compositing thread, 1 or 2 (see
        svr_batch_plan_set_pixels_per_thread); results do not depend on it
        beyond the order of gradient additions."""
        check(lib().svr_batch_plan_set_pixels_per_thread(self.plan, int(pixels)), "batch_plan_set_pixels_per_thread")
        self.pixels_per_thread = int(pixels)

    def set_backward_pixels_per_thread(self, pixels=None):
        """Pixels per thread of the backward alone, 1 or 2 (None: as
        set_pixels_per_thread)."""
        check(lib().svr_batch_plan_set_backward_pixels_per_thread(self.plan, int(pixels or 0)),
              "batch_plan_set_backward_pixels_per_thread")
        self.pixels_per_thread_bwd = int(pixels) if pixels else None

    def set_tile_size(self, tile_size, staging=None):
        """Compositing tile size (8, 16 or 32 pixels) and records staged per
        round (default 64 / 256 / 256).  A new tile size re-plans (the
        workspace and instance capacity change; call fit_capacity again)."""
        tile_size = int(tile_size)
        staging = int(staging) if staging is not None else (64 if tile_size == 8 else 256)
        if tile_size != self.tile_size:
            self.tile_size = tile_size
            self.staging = staging
            self.staging_bwd = None
            self._make_plan(self.capacity)
        else:
            self.set_staging(staging)

    def set_staging(self, records):
        """Records staged into shared memory per round, forward and backward
        (see svr_batch_plan_set_staging)."""
        check(lib().svr_batch_plan_set_staging(self.plan, int(records)), "batch_plan_set_staging")
        self.staging = int(records)
        self.staging_bwd = None

    def set_backward_staging(self, records=None):
        """The backward's staging depth alone (None: the forward's)."""
        r = self.staging if records is None else int(records)
        check(lib().svr_batch_plan_set_backward_staging(self.plan, r), "batch_plan_set_backward_staging")
        self.staging_bwd = None if records is None else r

    def set_sort_buckets(self, small_n=512, chunk=4096):
        """Segment-size buckets of the per-tile segment sort (small_n in
        256/512/1024, chunk in 2048/4096); the sorted order is the same for all."""
        self.sort_buckets = (int(small_n), int(chunk))
        check(lib().svr_batch_plan_set_sort_buckets(self.plan, *self.sort_buckets), "batch_plan_set_sort_buckets")

    def set_schedule(self, fwd_ordered=True, bwd_ordered=True, fwd_ctas_per_sm=0, bwd_ctas_per_sm=0):
        """Compositing schedule: per stage, tiles largest first (``*_ordered``)
        or in tile order, and caps on the resident CTAs per SM of the
        persistent forward / backward launches (0 = as many as fit).  Results
        do not depend on it."""
        self.schedule = (int(bool(fwd_ordered)) | (int(bool(bwd_ordered)) << 1), int(fwd_ctas_per_sm),
                         int(bwd_ctas_per_sm))
        check(lib().svr_batch_plan_set_schedule(self.plan, *self.schedule), "batch_plan_set_schedule")

    def __del__(self):
        try:
            if self.plan is not None:
                lib().svr_batch_plan_destroy(self.plan)
        except Exception:
            pass

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def _p(self, t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else None

    def header(self):
        """(total instance count, device error word) -- synchronises."""
        h = self.ws[:8].view(torch.int32).cpu()
        return int(h[0]) & 0xFFFFFFFF, int(h[1]) & 0xFFFFFFFF

    def fit_capacity(self, sh0, shs, sh_degree=3):
        """Run the projection + scan once, read the instance count and re-plan
        with `headroom` x that capacity (host sync; not for graph capture)."""
        self.prepare(sh0, shs, sh_degree)
        total, _ = self.header()
        need = int(math.ceil(total * self.headroom)) + 1024
        if need > self.capacity:
            self._make_plan(min(need, 0xFFFFFFFF))
        return total

    # -- stages ----------------------------------------------------------------
    def prepare(self, sh0, shs, sh_degree=3):
        bf16 = sh0.dtype == torch.bfloat16
        if bf16 != (shs.dtype == torch.bfloat16):
            raise ValueError("sh0 and shs must share a dtype")
        M = 1 + shs.shape[1]
        check(lib().svr_batch_prepare(self.plan, self._p(self.ws), self._p(self.octree_paths), self._p(self.centers),
                                      self._p(self.lengths), self._p(sh0.contiguous()),
                                      self._p(shs.contiguous()) if shs.numel() else None, int(bf16), int(sh_degree),
                                      M, self._stream()), "batch_prepare")

    def render(self, geos, out_color=None, out_T=None):
        """Composite every view; returns flat (color [sum 3HW], T [sum HW]).
        Every pixel of every view is written, so the outputs need no clearing."""
        if out_color is None:
            out_color = torch.empty(3 * self.n_pixels, device=self.dev)
            out_T = torch.empty(self.n_pixels, device=self.dev)
        check(lib().svr_batch_render(self.plan, self._p(self.ws), self._p(self.centers), self._p(self.lengths),
                                     self._p(geos), int(geos.dtype == torch.bfloat16), self._p(out_color),
                                     self._p(out_T), self._stream()), "batch_render")
        return out_color, out_T

    def backward(self, geos, out_T, dL_dcolor, dL_dT, sh_degree, M, grads=None):
        """Returns (dL_dgeos [P,8], subdiv [P], dL_dsh0 [P,3], dL_dshs [P,M-1,3]) fp32."""
        if grads is None:
            # dL_dgeos accumulates; subdiv and the SH gradients are overwritten
            grads = (torch.zeros(self.P, 8, device=self.dev), torch.empty(self.P, device=self.dev),
                     torch.empty(self.P, 3, device=self.dev), torch.empty(self.P, M - 1, 3, device=self.dev))
        else:
            grads[0].zero_()
        self.backward_render(geos, out_T, dL_dcolor, dL_dT, grads[0])
        self.backward_sh(sh_degree, M, grads[2], grads[3], grads[1])
        return grads

    def backward_render(self, geos, out_T, dL_dcolor, dL_dT, dL_dgeos):
        """The compositing backward alone: adds every view's density gradient
        into dL_dgeos [P,8] (16-byte aligned) and keeps the per-view colour
        gradients in the workspace for backward_sh."""
        check(lib().svr_batch_backward(self.plan, self._p(self.ws), self._p(self.centers), self._p(self.lengths),
                                       self._p(geos), int(geos.dtype == torch.bfloat16), self._p(out_T),
                                       self._p(dL_dcolor), self._p(dL_dT), self._p(dL_dgeos), self._stream()),
              "batch_backward")

    def render_grid(self, vox_key, grid_pts, out_color=None, out_T=None):
        """render() with grid-point densities read while staging: corner c of
        voxel p is grid_pts[vox_key[p, c]] (vox_key int64 [P,8], grid fp32 or
        bf16).  Same outputs as gather_grid_geos + render."""
        if out_color is None:
            out_color = torch.empty(3 * self.n_pixels, device=self.dev)
            out_T = torch.empty(self.n_pixels, device=self.dev)
        check(lib().svr_batch_render_grid(self.plan, self._p(self.ws), self._p(self.centers), self._p(self.lengths),
                                          self._p(vox_key), self._p(grid_pts), int(grid_pts.dtype == torch.bfloat16),
                                          self._p(out_color), self._p(out_T), self._stream()), "batch_render_grid")
        return out_color, out_T

    def backward_render_grid(self, vox_key, grid_pts, out_T, dL_dcolor, dL_dT, dL_dgrid):
        """backward_render() adding each record's corner gradients straight
        into dL_dgrid [M] fp32 (accumulates; zero it first)."""
        check(lib().svr_batch_backward_grid(self.plan, self._p(self.ws), self._p(self.centers), self._p(self.lengths),
                                            self._p(vox_key), self._p(grid_pts),
                                            int(grid_pts.dtype == torch.bfloat16), self._p(out_T),
                                            self._p(dL_dcolor), self._p(dL_dT), self._p(dL_dgrid), self._stream()),
              "batch_backward_grid")

    def backward_sh(self, sh_degree, M, dL_dsh0, dL_dshs, subdiv=None):
        """SH gradients (and the subdivision priority) summed over views, from
        the colour gradients of the last backward_render (overwritten)."""
        check(lib().svr_batch_sh_backward(self.plan, self._p(self.ws), self._p(self.centers), int(sh_degree), int(M),
                                          self._p(dL_dsh0), self._p(dL_dshs) if dL_dshs.numel() else None,
                                          self._p(subdiv), self._stream()), "batch_sh_backward")

    # -- views of the flat outputs ---------------------------------------------
    def split_color(self, flat):
        return [flat[3 * a:3 * b].view(3, h, w) for (h, w), a, b in
                zip(self.sizes, self.pix_offsets[:-1], self.pix_offsets[1:])]

    def split_pixels(self, flat):
        return [flat[a:b].view(1, h, w) for (h, w), a, b in zip(self.sizes, self.pix_offsets[:-1],
                                                                 self.pix_offsets[1:])]

    def arrays(self):
        """Device views of the workspace internals (rgbs, n_contrib, ...)."""
        ptrs = [ctypes.c_void_p() for _ in range(7)]
        check(lib().svr_batch_arrays(self.plan, self._p(self.ws), *[ctypes.byref(p) for p in ptrs]), "arrays")
        base = self.ws.data_ptr()
        off = [p.value - base for p in ptrs]
        VP = len(self.cams) * self.P
        ws = self.ws
        ob = lib().svr_batch_bbox_ptr(self.plan, self._p(self.ws)) - base
        return dict(
            bbox=ws[ob:ob + 8 * VP].view(torch.int32).view(len(self.cams), self.P, 2),
            rgbs=ws[off[0]:off[0] + 12 * VP].view(torch.float32).view(len(self.cams), self.P, 3),
            drgbs=ws[off[1]:off[1] + 16 * VP].view(torch.float32).view(len(self.cams), self.P, 4),
            ranges=ws[off[2]:off[2] + 8 * self.n_tiles].view(torch.int32).view(self.n_tiles, 2),
            tile_last=ws[off[3]:off[3] + 4 * self.n_tiles].view(torch.int32),
            n_contrib=ws[off[4]:off[4] + 4 * self.n_pixels].view(torch.int32),
            ndup=ws[off[5]:off[5] + 4 * VP].view(torch.int32).view(len(self.cams), self.P),
            sorted_vals=ws[off[6]:off[6] + 4 * max(self.capacity, 1)].view(torch.int32),
        )


class BatchedRender(torch.autograd.Function):
    """Autograd wrapper: (geos, sh0, shs) -> (color flat, T flat) over all views."""

    @staticmethod
    def forward(ctx, raster, sh_degree, geos, sh0, shs):
        raster.prepare(sh0, shs, sh_degree)
        color, T = raster.render(geos)
        ctx.raster = raster
        ctx.sh_degree = sh_degree
        ctx.M = 1 + shs.shape[1]
        ctx.sh_dtype = sh0.dtype
        ctx.save_for_backward(geos, T)
        return color, T

    @staticmethod
    def backward(ctx, dL_dcolor, dL_dT):
        geos, T = ctx.saved_tensors
        r = ctx.raster
        if dL_dT is None:
            dL_dT = torch.zeros_like(T)
        dgeo, _sub, dsh0, dshs = r.backward(geos, T, dL_dcolor.contiguous(), dL_dT.contiguous(), ctx.sh_degree, ctx.M)
        return None, None, dgeo.to(geos.dtype), dsh0.to(ctx.sh_dtype), dshs.to(ctx.sh_dtype)


def gather_grid_geos(vox_key, grid_pts, out):
    """out[p, c] = grid_pts[vox_key[p, c]] for every voxel (GatherGeoParams
    with all voxels cared for; grid and out fp32 or bf16)."""
    P = vox_key.shape[0]
    check(lib().svr_gather_grid_geo_all(P, ctypes.c_void_p(vox_key.data_ptr()), ctypes.c_void_p(grid_pts.data_ptr()),
                                        int(grid_pts.dtype == torch.bfloat16), ctypes.c_void_p(out.data_ptr()),
                                        int(out.dtype == torch.bfloat16),
                                        ctypes.c_void_p(torch.cuda.current_stream(out.device).cuda_stream)),
          "gather_grid_geo_all")
    return out


def scatter_grid_grad(vox_key, dL_dgeos, dL_dgrid):
    """dL_dgrid[vox_key[p, c]] += dL_dgeos[p, c] (fp32) for every voxel."""
    P = vox_key.shape[0]
    check(lib().svr_scatter_grid_geo_all(P, ctypes.c_void_p(vox_key.data_ptr()), ctypes.c_void_p(dL_dgeos.data_ptr()),
                                         ctypes.c_void_p(dL_dgrid.data_ptr()),
                                         ctypes.c_void_p(torch.cuda.current_stream(dL_dgrid.device).cuda_stream)),
          "scatter_grid_geo_all")
    return dL_dgrid


class GridBatchedRender(torch.autograd.Function):
    """Autograd wrapper over grid-point densities, the reference's training
    parametrisation (GatherGeoParams then rasterize, renderer.py:319-345):
    (grid_pts [M], sh0, shs) -> (color flat, T flat) over all views.  The
    corner densities are gathered once per step for all views into a [P,8]
    buffer of the grid's dtype, and the density gradients are added back into
    the grid gradient once per step.  With ``fused=True`` the compositing
    kernels read the grid points while staging each record and add the
    corner gradients into the grid gradient in their flush instead (no [P,8]
    buffer; per (voxel, tile) grid accesses instead of per voxel -- measured
    3 % slower at one view per step and 8 % slower at eight, see
    svr_batch_render_grid)."""

    @staticmethod
    def forward(ctx, raster, sh_degree, vox_key, grid_pts, sh0, shs, fused=False):
        raster.prepare(sh0, shs, sh_degree)
        if fused:
            geos = None
            color, T = raster.render_grid(vox_key, grid_pts)
            ctx.save_for_backward(vox_key, grid_pts, T)
        else:
            geos = torch.empty(vox_key.shape[0], 8, dtype=grid_pts.dtype, device=grid_pts.device)
            gather_grid_geos(vox_key, grid_pts, geos)
            color, T = raster.render(geos)
            ctx.save_for_backward(vox_key, geos, T)
        ctx.raster, ctx.sh_degree, ctx.M, ctx.fused = raster, sh_degree, 1 + shs.shape[1], bool(fused)
        ctx.sh_dtype, ctx.grid_dtype, ctx.M_grid = sh0.dtype, grid_pts.dtype, grid_pts.shape[0]
        return color, T

    @staticmethod
    def backward(ctx, dL_dcolor, dL_dT):
        vox_key, dens, T = ctx.saved_tensors
        r = ctx.raster
        if dL_dT is None:
            dL_dT = torch.zeros_like(T)
        dgrid = torch.zeros(ctx.M_grid, dtype=torch.float32, device=T.device)
        P, M = vox_key.shape[0], ctx.M
        if ctx.fused:
            r.backward_render_grid(vox_key, dens, T, dL_dcolor.contiguous(), dL_dT.contiguous(), dgrid)
            dsh0 = torch.empty(P, 3, device=T.device)
            dshs = torch.empty(P, M - 1, 3, device=T.device)
            r.backward_sh(ctx.sh_degree, M, dsh0, dshs)
        else:
            dgeo, _sub, dsh0, dshs = r.backward(dens, T, dL_dcolor.contiguous(), dL_dT.contiguous(), ctx.sh_degree, M)
            scatter_grid_grad(vox_key, dgeo, dgrid)
        return (None, None, None, dgrid.to(ctx.grid_dtype), dsh0.to(ctx.sh_dtype), dshs.to(ctx.sh_dtype), None)
