// Backward compositing of one tile with each lane walking its own pixel's
// records ("lane form"), for the batched 8x8 configurations.
//
// The warp-synchronous form (render_tile_bwd) visits every staged record
// that touches the warp's 8x4 pixels with all 32 lanes, so a record reached
// by a few pixels costs the whole warp the recomputed quadrature, and its
// gradients are reduced across the warp record by record.  Here, per group
// of 32 staged records and per warp:
//
//   1. candidate masks: for each record touching the warp, the ballot of
//      lanes whose pixel lies in its bbox with a matching quadrant and whose
//      contributor range reaches it (cm[r]), and per lane the mask of its
//      own records; each record's candidate (record, pixel) pairs get
//      consecutive row slots (record-major, exclusive scan of popc(cm));
//   2. walk: every lane steps through its own records in back-to-front
//      order (bwd_pixel_record: the same per-(pixel, record) arithmetic as
//      the warp-synchronous form) and writes the 12 gradient values of each
//      candidate pair into that pair's row (zeros when it does not
//      contribute) -- a warp takes as many iterations as its busiest pixel
//      has records, not one per record;
//   3. sums: lanes take (record, column) tasks and add the record's rows of
//      that column, storing the warp's total into its per-record slot.
//
// Rows are bounded by kLaneRows per warp: a group whose pairs exceed it is
// processed in sub-groups of consecutive records (a record's pairs never
// exceed 32).  A pixel's records stay in order across sub-groups and
// groups, so its transmittance recovery and running sums see the same
// sequence as the warp-synchronous form; only the order of the gradient
// additions differs.  The flush is the warp-synchronous form's: one set of
// global reductions per (voxel, tile) with the two warps' slots summed.
#pragma once

#include "svr_render_bwd.cuh"

namespace svr {

constexpr int kLaneRows = 64;  // (record, pixel) gradient rows per warp and sub-group

template <class CFG>
struct LaneBwdSmem {
  static_assert(CFG::TS == 8 && CFG::NW == 2, "the lane form serves 8x8 tiles (two warps of 8x4 pixels)");
  float acc[CFG::NW][CFG::SB][12];   // per-warp record totals of this staging round
  float rows[CFG::NW][kLaneRows][12];
  uint32_t cm[CFG::NW][32];          // candidate lanes of each record of the current group
  uint32_t off[CFG::NW][33];         // first row of each record (exclusive scan), [32] = total
  uint32_t wrote[CFG::NW][CFG::GROUPS];
};

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <class CFG, int NS, bool FAST = false, bool RGB4 = false>
__device__ __forceinline__ void render_tile_bwd_lanes(const ViewParams& vp, const float* __restrict__ c2w_s,
                                                      int tile_x, int tile_y, uint2 range_raw, uint32_t tile_last,
                                                      const uint32_t* __restrict__ vals, const VoxelArrays& va,
                                                      const BwdTileIn& in, const BwdTileOut& out,
                                                      StageSmem<CFG::SB>& s, LaneBwdSmem<CFG>& L) {
  constexpr int SB = CFG::SB;
  const int W = vp.W, H = vp.H;
  const int tid = threadIdx.x, lane = tid & 31;
  int lx, ly;
  tile_pixel_of<CFG>(tid, lx, ly);
  const uint32_t px = tile_x * CFG::TS + lx, py = tile_y * CFG::TS + ly;
  const uint32_t pix_id = (uint32_t)W * py + px;
  const bool inside = px < (uint32_t)W && py < (uint32_t)H;
  const PixelRay ray = make_pixel_ray((float)px, (float)py, W, H, vp.tanfovx, vp.tanfovy, vp.cx, vp.cy, c2w_s);
  const int warp = tid >> 5;
  const uint32_t wx0 = tile_x * CFG::TS + (warp % CFG::MX) * 8, wy0 = tile_y * CFG::TS + (warp / CFG::MX) * 4;

  // Range check (replaces the __trap at backward.cu:122-133).
  if (tile_last > range_raw.y || range_raw.x > tile_last) {
    if (tid == 0) atomicOr(out.err, SVR_DEVERR_RANGE);
    return;
  }
  const uint2 range = make_uint2(range_raw.x, tile_last);
  const float T_final = inside ? in.T[pix_id] : 0.f;
  const int todo_total = (int)(range.y - range.x);
  const uint32_t last_contrib = inside ? in.n_contrib[pix_id] : 0u;
  BwdPix st = bwd_pixel_init<false, false, false>(vp, in, ray, inside, pix_id, T_final);
  const uint32_t warp_lc = __reduce_max_sync(0xffffffffu, last_contrib);
  const uint32_t quad_mask = __reduce_or_sync(0xffffffffu, inside ? (1u << ray.quad) : 0u);
  const uint32_t below = lanemask_lt();
  float(*rows)[12] = L.rows[warp];
  uint32_t* cm_s = L.cm[warp];
  uint32_t* off_s = L.off[warp];

  const int rounds = (todo_total + SB - 1) / SB;
  for (int r = 0; r < rounds; ++r) {
    __syncthreads();
    const int base = r * SB;  // records [base, base+n_here) from the back
    const int n_here = min(SB, todo_total - base);
    for (int i = tid; i < n_here; i += CFG::NT)
      stage_record(s, i, vals[range.y - base - i - 1], va, ray.ox, ray.oy, ray.oz);
    __syncthreads();

    for (int g = 0; g < CFG::GROUPS; ++g) {
      uint32_t wrote = 0u;
      if (g * 32 < n_here) {
        // Position (relative to range.x) of staged slot j is todo_total - base - j - 1.
        const int slot = g * 32 + lane;
        const uint32_t pos = (uint32_t)(todo_total - base - slot - 1);
        const bool hit = slot < n_here && pos < warp_lc && record_hits_warp(s, slot, wx0, wy0, quad_mask);
        uint32_t m = __ballot_sync(0xffffffffu, hit);
        // 1. candidate masks: lane b keeps record b's, every lane its own records
        uint32_t my_cm = 0u, mine = 0u;
        while (m) {
          const int b = __ffs(m) - 1;
          m &= m - 1;
          const int j = g * 32 + b;
          const uint32_t jpos = (uint32_t)(todo_total - base - j - 1);
          const bool c = inside && jpos < last_contrib && record_hits_pixel(s, j, px, py, ray.quad);
          const uint32_t cm = __ballot_sync(0xffffffffu, c);
          if (lane == b) my_cm = cm;
          mine |= (uint32_t)c << b;
        }
        const uint32_t cnt = __popc(my_cm);
        uint32_t incl = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
          if (lane >= d) incl += t;
        }
        const uint32_t my_off = incl - cnt;
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        cm_s[lane] = my_cm;
        off_s[lane] = my_off;
        if (lane == 0) off_s[32] = total;
        wrote = __ballot_sync(0xffffffffu, cnt > 0u);
        __syncwarp();
        // sub-groups of consecutive records whose rows fit
        int b0 = 0;
        while (b0 < 32) {
          const uint32_t row0 = __shfl_sync(0xffffffffu, my_off, b0);
          if (row0 == total) break;
          const bool fits = lane < b0 || my_off + cnt - row0 <= (uint32_t)kLaneRows;
          const int b1 = __popc(__ballot_sync(0xffffffffu, fits));  // fits holds on a prefix of lanes
          const uint32_t sub = (b1 == 32 ? 0xffffffffu : ((1u << b1) - 1u)) & ~((1u << b0) - 1u);
          // 2. walk: this lane's records of the sub-group, back to front
          uint32_t my = mine & sub;
          while (my) {
            const int b = __ffs(my) - 1;
            my &= my - 1;
            float gp[12];
            const bool contrib = bwd_pixel_record<SB, NS, false, false, false, FAST>(s, g * 32 + b, ray, in, st, gp);
            const uint32_t row = off_s[b] - row0 + __popc(cm_s[b] & below);
            float4* r4 = reinterpret_cast<float4*>(rows[row]);
            if (contrib) {
              r4[0] = make_float4(gp[0], gp[1], gp[2], gp[3]);
              r4[1] = make_float4(gp[4], gp[5], gp[6], gp[7]);
              r4[2] = make_float4(gp[8], gp[9], gp[10], gp[11]);
            } else {
              const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
              r4[0] = z; r4[1] = z; r4[2] = z;
            }
          }
          __syncwarp();
          // 3. sums: task t = (record b0 + t / 12, column t % 12)
          const int n_tasks = 12 * (b1 - b0);
          for (int t = lane; t < n_tasks; t += 32) {
            const int b = b0 + t / 12, c = t - (t / 12) * 12;
            const uint32_t o = off_s[b] - row0, n = off_s[b + 1] - off_s[b];
            if (n == 0u) continue;
            float sum = 0.f;
            for (uint32_t i = 0; i < n; ++i) sum += rows[o + i][c];
            L.acc[warp][g * 32 + b][c] = sum;
          }
          __syncwarp();  // the rows are rewritten by the next sub-group
          b0 = b1;
        }
      }
      if (lane == 0) L.wrote[warp][g] = wrote;
    }
    __syncthreads();
    // Flush this batch's accumulators: one set of reductions per (voxel, tile).
    for (int t = tid; t < n_here; t += CFG::NT) {
      float acc[12];
#pragma unroll
      for (int c = 0; c < 12; ++c) acc[c] = 0.f;
      bool any = false;
#pragma unroll
      for (int w = 0; w < CFG::NW; ++w) {
        if (!((L.wrote[w][t >> 5] >> (t & 31)) & 1u)) continue;
        any = true;
        const float4* a4 = reinterpret_cast<const float4*>(L.acc[w][t]);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const float4 v = a4[q];
          acc[4 * q] += v.x; acc[4 * q + 1] += v.y; acc[4 * q + 2] += v.z; acc[4 * q + 3] += v.w;
        }
      }
      if (!any) continue;
      float gsum = 0.f;
#pragma unroll
      for (int c = 0; c < 12; ++c) gsum += fabsf(acc[c]);
      if (gsum != 0.f) {
        const uint32_t vid = (uint32_t)__float_as_int(s.corner[t].w);
        float* gdst = out.dL_dgeos + 8 * (size_t)vid;
        if (RGB4 || out.geo_vec4) {
          atomicAdd(reinterpret_cast<float4*>(gdst), make_float4(acc[0], acc[1], acc[2], acc[3]));
          atomicAdd(reinterpret_cast<float4*>(gdst) + 1, make_float4(acc[4], acc[5], acc[6], acc[7]));
        } else {
#pragma unroll
          for (int c = 0; c < 8; ++c) atomicAdd(gdst + c, acc[c]);
        }
        if (RGB4) {
          atomicAdd(reinterpret_cast<float4*>(out.dL_drgbs) + vid, make_float4(acc[8], acc[9], acc[10], acc[11]));
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) atomicAdd(out.dL_drgbs + 3 * (size_t)vid + c, acc[8 + c]);
          atomicAdd(out.subdiv + vid, acc[11]);
        }
      }
    }
  }
}

}  // namespace svr
