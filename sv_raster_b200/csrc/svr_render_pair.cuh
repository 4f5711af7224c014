// Compositing with two pixels per thread (batched path, colour and
// transmittance only).
//
// A warp covers an 8x8 block of the tile: lane l owns the pixels
// (l & 7, l >> 3) and (l & 7, (l >> 3) + 4).  A staged record that a warp's
// ballot selects is tested against both pixels; the records' shared-memory
// fields are read once for the pair, and in the backward the two pixels'
// gradients are added in registers before the one warp reduction of the
// record.  With one pixel per thread the same 8x8 block is two warps, and a
// record touching both halves costs two ballots, two sets of loads and two
// reductions.
//
// The per-pixel arithmetic is the one of svr_render_fwd.cuh /
// svr_render_bwd.cuh (forward.cu:182-316, backward.cu:246-418) without the
// depth, distortion, normal and regulariser terms, expression for expression,
// so images, T and contributor counts equal the one-pixel kernels' bit for
// bit; gradients differ only in the order of additions.
#pragma once

#include "svr_render_bwd.cuh"
#include "svr_render_fwd.cuh"

namespace svr {

// TS x TS tiles, TS*TS/2 threads, warps laid out row-major as 8x8 blocks,
// SB records staged per round.
template <int TS_, int SB_>
struct PairCfg {
  static constexpr int TS = TS_;
  static constexpr int NT = TS * TS / 2;  // threads per CTA
  static constexpr int NW = NT / 32;      // warps per CTA
  static constexpr int MX = TS / 8;       // 8x8 blocks per tile row
  static constexpr int SB = SB_;
  static constexpr int GROUPS = SB / 32;
  static_assert(TS == 8 || TS == 16, "tile size");
  static_assert(SB % 32 == 0 && SB >= 32, "staging depth");
};

// Resident CTAs per SM the pair kernels are register-bounded for, per 32
// threads: 20 warps of 32 threads leave each thread about 100 registers for
// the two pixels' state.
constexpr int kPairWarpsPerSM = 20;
template <class CFG>
constexpr int pair_min_blocks() { return kPairWarpsPerSM / CFG::NW; }

// Does staged record `slot` possibly touch a pixel of this warp's 8x8 block
// with a matching ray quadrant?
template <int SB>
__device__ __forceinline__ bool record_hits_block8(const StageSmem<SB>& s, int slot, uint32_t wx0, uint32_t wy0,
                                                   uint32_t quad_mask) {
  const uint4 b = s.box[slot];
  return b.x <= wx0 + 7u && b.x + b.y >= wx0 && b.z <= wy0 + 7u && b.z + (b.w & 0xFFFFu) >= wy0 &&
         ((quad_mask >> (b.w >> 16)) & 1u);
}

// Optical depth of the ray segment [a, b] through staged record j
// (forward.cu:228-248): midpoint samples of the activated trilinear density.
template <int NS, bool FAST, int SB>
__device__ __forceinline__ float record_vol_int(const StageSmem<SB>& s, int j, const PixelRay& ray, float a, float b,
                                                float vox_l_inv) {
  float geo[8];
  load_geo(s, j, geo);
  float vol_int = 0.f;
  float w[8];
  const float4 cr = s.corner[j];
  const float step_sz = (b - a) * (1.f / NS);
  const float stx = step_sz * ray.dx, sty = step_sz * ray.dy, stz = step_sz * ray.dz;
  const float t0 = a + 0.5f * step_sz;
  const float ptx = ray.ox + t0 * ray.dx, pty = ray.oy + t0 * ray.dy, ptz = ray.oz + t0 * ray.dz;
  float qx = (ptx - cr.x) * vox_l_inv;
  float qy = (pty - cr.y) * vox_l_inv;
  float qz = (ptz - cr.z) * vox_l_inv;
  const float qsx = stx * vox_l_inv, qsy = sty * vox_l_inv, qsz = stz * vox_l_inv;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    trilinear_weights(qx, qy, qz, w);
    float d = 0.f;
#pragma unroll
    for (int c = 0; c < 8; ++c) d += geo[c] * w[c];
    const float lvi = kStepScale * step_sz * density_act_f<FAST>(d);
    vol_int += lvi;
    qx = qx + qsx; qy = qy + qsy; qz = qz + qsz;
  }
  return vol_int;
}

template <class CFG, int NS, bool FAST>
__device__ __forceinline__ void render_tile_fwd_pair(const ViewParams& vp, const float* __restrict__ c2w_s,
                                                     int tile_x, int tile_y, uint2 range,
                                                     const uint32_t* __restrict__ vals, const VoxelArrays& va,
                                                     const FwdTileOut& out, uint32_t* last_slot,
                                                     StageSmem<CFG::SB>& s, uint32_t* s_red /*[CFG::NW]*/) {
  constexpr int SB = CFG::SB;
  const int W = vp.W, H = vp.H;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t wx0 = tile_x * CFG::TS + (warp % CFG::MX) * 8, wy0 = tile_y * CFG::TS + (warp / CFG::MX) * 8;
  const uint32_t px = wx0 + (lane & 7);
  uint32_t py[2];
  bool inside[2], done[2];
  PixelRay ray[2];
  float T[2], Cx[2], Cy[2], Cz[2];
  uint32_t last_contrib[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    py[k] = wy0 + (lane >> 3) + 4 * k;
    inside[k] = px < (uint32_t)W && py[k] < (uint32_t)H;
    ray[k] = make_pixel_ray((float)px, (float)py[k], W, H, vp.tanfovx, vp.tanfovy, vp.cx, vp.cy, c2w_s);
    done[k] = !inside[k];
    T[k] = 1.f;
    Cx[k] = Cy[k] = Cz[k] = 0.f;
    last_contrib[k] = 0;
  }

  const int todo_total = (int)(range.y - range.x);
  const int rounds = (todo_total + SB - 1) / SB;
  for (int r = 0; r < rounds; ++r) {
    if (__syncthreads_count(done[0] && done[1]) == CFG::NT) break;
    const int base = r * SB;
    const int n_here = min(SB, todo_total - base);
    for (int i = tid; i < n_here; i += CFG::NT)
      stage_record(s, i, vals[range.x + base + i], va, ray[0].ox, ray[0].oy, ray[0].oz);
    __syncthreads();

    const uint32_t quad_mask = __reduce_or_sync(
        0xffffffffu, (done[0] ? 0u : (1u << ray[0].quad)) | (done[1] ? 0u : (1u << ray[1].quad)));
    if (quad_mask == 0u) continue;
    for (int g = 0; g < CFG::GROUPS && g * 32 < n_here; ++g) {
      const int slot = g * 32 + lane;
      const bool hit = slot < n_here && record_hits_block8(s, slot, wx0, wy0, quad_mask);
      uint32_t m = __ballot_sync(0xffffffffu, hit);
      while (m) {
        const int j = g * 32 + __ffs(m) - 1;
        m &= m - 1;
        const float4 slo = s.slab_lo[j], shi = s.slab_hi[j];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          if (done[k] || !record_hits_pixel(s, j, px, py[k], ray[k].quad)) continue;
          const float2 ab = staged_ray_box(slo, shi, ray[k]);
          const float a = ab.x, b = ab.y;
          if (a > b) continue;
          const float vol_int = record_vol_int<NS, FAST>(s, j, ray[k], a, b, slo.w);
          const float alpha = fminf(kMaxAlpha, 1.f - exp_f<FAST>(-vol_int));
          if (alpha < kMinAlpha) continue;
          const float pt_w = T[k] * alpha;
          const float4 rgbv = s.rgb[j];
          Cx[k] = Cx[k] + pt_w * rgbv.x;
          Cy[k] = Cy[k] + pt_w * rgbv.y;
          Cz[k] = Cz[k] + pt_w * rgbv.z;
          T[k] *= (1.f - alpha);
          done[k] |= (T[k] < kEarlyStopT);
          last_contrib[k] = (uint32_t)(base + j + 1);
        }
      }
    }
  }

  const size_t HW = (size_t)H * W;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    if (!inside[k]) continue;
    const uint32_t pix_id = (uint32_t)W * py[k] + px;
    out.n_contrib[pix_id] = last_contrib[k];
    out.color[0 * HW + pix_id] = Cx[k] + T[k] * vp.bg;
    out.color[1 * HW + pix_id] = Cy[k] + T[k] * vp.bg;
    out.color[2 * HW + pix_id] = Cz[k] + T[k] * vp.bg;
    out.T[pix_id] = T[k];
  }
  const uint32_t mine = max(inside[0] ? last_contrib[0] : 0u, inside[1] ? last_contrib[1] : 0u);
  const uint32_t lc = __reduce_max_sync(0xffffffffu, mine);
  if (lane == 0) s_red[warp] = lc;
  __syncthreads();
  if (tid == 0) {
    uint32_t mx = 0;
#pragma unroll
    for (int w = 0; w < CFG::NW; ++w) mx = max(mx, s_red[w]);
    *last_slot = range.x + mx;
  }
}

// GRID: densities as grid points (VoxelArrays::key / BwdTileOut::key set);
// the per-voxel form is instantiated without the grid reads.
template <class CFG, int NS, bool FAST, bool GRID = false>
__device__ __forceinline__ void render_tile_bwd_pair(const ViewParams& vp, const float* __restrict__ c2w_s,
                                                     int tile_x, int tile_y, uint2 range_raw, uint32_t tile_last,
                                                     const uint32_t* __restrict__ vals, const VoxelArrays& va,
                                                     const BwdTileIn& in, const BwdTileOut& out,
                                                     StageSmem<CFG::SB>& s, float* s_grad /*[GradAcc::kFloats]*/,
                                                     uint32_t* s_hit /*[GradAcc::kWords]*/) {
  using Acc = GradAcc<CFG>;
  constexpr int SB = CFG::SB;
  const int W = vp.W, H = vp.H;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t wx0 = tile_x * CFG::TS + (warp % CFG::MX) * 8, wy0 = tile_y * CFG::TS + (warp / CFG::MX) * 8;
  const uint32_t px = wx0 + (lane & 7);

  // Range check (replaces the __trap at backward.cu:122-133).
  if (tile_last > range_raw.y || range_raw.x > tile_last) {
    if (tid == 0) atomicOr(out.err, SVR_DEVERR_RANGE);
    return;
  }
  const uint2 range = make_uint2(range_raw.x, tile_last);
  const size_t HW = (size_t)H * W;
  const int todo_total = (int)(range.y - range.x);

  uint32_t py[2], last_contrib[2];
  bool inside[2];
  PixelRay ray[2];
  float T[2], gx[2], gy[2], gz[2], last_dL_dT[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    py[k] = wy0 + (lane >> 3) + 4 * k;
    inside[k] = px < (uint32_t)W && py[k] < (uint32_t)H;
    ray[k] = make_pixel_ray((float)px, (float)py[k], W, H, vp.tanfovx, vp.tanfovy, vp.cx, vp.cy, c2w_s);
    const uint32_t pix_id = (uint32_t)W * py[k] + px;
    T[k] = inside[k] ? in.T[pix_id] : 0.f;
    last_contrib[k] = inside[k] ? in.n_contrib[pix_id] : 0u;
    gx[k] = gy[k] = gz[k] = last_dL_dT[k] = 0.f;
    if (inside[k]) {
      gx[k] = in.dL_dcolor[0 * HW + pix_id];
      gy[k] = in.dL_dcolor[1 * HW + pix_id];
      gz[k] = in.dL_dcolor[2 * HW + pix_id];
      last_dL_dT[k] = in.dL_dT[pix_id] + vp.bg * (gx[k] + gy[k] + gz[k]);
    }
  }

  Acc::init(s_grad, tid);
  const uint32_t warp_lc = __reduce_max_sync(0xffffffffu, max(last_contrib[0], last_contrib[1]));
  const uint32_t quad_mask = __reduce_or_sync(
      0xffffffffu, (inside[0] ? (1u << ray[0].quad) : 0u) | (inside[1] ? (1u << ray[1].quad) : 0u));
  // Lane q holds, per pixel row k, the lanes whose pixel k is in the image
  // with ray quadrant q.
  uint32_t qlanes[2] = {0u, 0u};
  for (uint32_t qm = quad_mask; qm; qm &= qm - 1) {
    const uint32_t q = (uint32_t)(__ffs(qm) - 1);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const uint32_t bk = __ballot_sync(0xffffffffu, inside[k] && ray[k].quad == q);
      if ((uint32_t)lane == q) qlanes[k] = bk;
    }
  }

  const int rounds = (todo_total + SB - 1) / SB;
  for (int r = 0; r < rounds; ++r) {
    __syncthreads();
    const int base = r * SB;
    const int n_here = min(SB, todo_total - base);
    for (int i = tid; i < n_here; i += CFG::NT)
      stage_record<CFG::SB, GRID>(s, i, vals[range.y - base - i - 1], va, ray[0].ox, ray[0].oy, ray[0].oz);
    __syncthreads();

    for (int g = 0; g < CFG::GROUPS && g * 32 < n_here; ++g) {
      const int slot = g * 32 + lane;
      const uint32_t pos = (uint32_t)(todo_total - base - slot - 1);
      const bool hit = slot < n_here && pos < warp_lc && record_hits_block8(s, slot, wx0, wy0, quad_mask);
      uint32_t m = __ballot_sync(0xffffffffu, hit);
      // Each lane's candidate records of this group per pixel: lane j turns
      // record j's bbox into masks of the pixels it covers in the two 8x4
      // halves, restricted to the lanes of its ray quadrant, and a bit
      // transposition hands every lane its records; a record reaches pixel k
      // only while its position is below the pixel's contributor count.
      uint32_t cov[2] = {0u, 0u};
      uint32_t rec_quad = 0u;
      if (hit) {
        const uint4 b = s.box[slot];
        cov[0] = block_cover_mask(b, wx0, wy0);
        cov[1] = block_cover_mask(b, wx0, wy0 + 4u);
        rec_quad = b.w >> 16;
      }
      uint32_t mine[2];
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        mine[k] = warp_transpose_bits(cov[k] & __shfl_sync(0xffffffffu, qlanes[k], (int)rec_quad), (uint32_t)lane);
        // slot j is in reach while todo_total - base - j - 1 < last_contrib[k]
        const int first = todo_total - base - (int)last_contrib[k] - g * 32;
        mine[k] &= first <= 0 ? 0xffffffffu : (first >= 32 ? 0u : ~((1u << first) - 1u));
      }
      m &= __reduce_or_sync(0xffffffffu, mine[0] | mine[1]);  // records no pixel of the warp takes
      uint32_t wrote = 0u;
      while (m) {
        const int bit = __ffs(m) - 1;
        const int j = g * 32 + bit;
        m &= m - 1;
        float gp[12];
#pragma unroll
        for (int c = 0; c < 12; ++c) gp[c] = 0.f;
        bool contrib = false;
        const float4 slo = s.slab_lo[j], shi = s.slab_hi[j];
        // the record's densities and corner, read once for both pixels
        float geo[8];
        load_geo(s, j, geo);
        const float4 cr = s.corner[j];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          if (!((mine[k] >> bit) & 1u)) continue;
          const float2 ab = staged_ray_box(slo, shi, ray[k]);
          const float a = ab.x, b = ab.y;
          if (a > b) continue;
          float vol_int = 0.f;
          float dI_dgeo[8];
#pragma unroll
          for (int c = 0; c < 8; ++c) dI_dgeo[c] = 0.f;
          float w[8];
          const float vox_l_inv = slo.w;
          const float step_sz = (b - a) * (1.f / NS);
          const float stx = step_sz * ray[k].dx, sty = step_sz * ray[k].dy, stz = step_sz * ray[k].dz;
          const float t0 = a + 0.5f * step_sz;
          const float ptx = ray[k].ox + t0 * ray[k].dx, pty = ray[k].oy + t0 * ray[k].dy,
                      ptz = ray[k].oz + t0 * ray[k].dz;
          float qx = (ptx - cr.x) * vox_l_inv;
          float qy = (pty - cr.y) * vox_l_inv;
          float qz = (ptz - cr.z) * vox_l_inv;
          const float qsx = stx * vox_l_inv, qsy = sty * vox_l_inv, qsz = stz * vox_l_inv;
#pragma unroll
          for (int n = 0; n < NS; ++n) {
            trilinear_weights(qx, qy, qz, w);
            float d = 0.f;
#pragma unroll
            for (int c = 0; c < 8; ++c) d += geo[c] * w[c];
            float act, act_grad;
            density_act_and_grad_f<FAST>(d, act, act_grad);
            const float lvi = kStepScale * step_sz * act;
            vol_int += lvi;
            const float dd_dd = kStepScale * step_sz * act_grad;
            if (FAST && NS == 1) {
              dI_dgeo[0] = dd_dd;  // the weights stay in w: dL/dgeo = (dL/dI * dd_dd) * w below
            } else {
#pragma unroll
              for (int c = 0; c < 8; ++c) dI_dgeo[c] += dd_dd * w[c];
            }
            qx = qx + qsx; qy = qy + qsy; qz = qz + qsz;
          }
          const float exp_neg = exp_f<FAST>(-vol_int);
          const float alpha = fminf(kMaxAlpha, 1.f - exp_neg);
          if (alpha < kMinAlpha) continue;
          contrib = true;
          T[k] = div_f<FAST>(T[k], 1.f - alpha);
          const float pt_w = alpha * T[k];
          const float4 rgbv = s.rgb[j];
          const float dL_dpt_w = gx[k] * rgbv.x + gy[k] * rgbv.y + gz[k] * rgbv.z;
          const float dL_dalpha = T[k] * (dL_dpt_w - last_dL_dT[k]);
          last_dL_dT[k] += alpha * (dL_dpt_w - last_dL_dT[k]);
          const float dL_dI = dL_dalpha * exp_neg;
          if (FAST && NS == 1) {
            const float sI = dL_dI * dI_dgeo[0];
#pragma unroll
            for (int c = 0; c < 8; ++c) gp[c] += sI * w[c];
          } else {
#pragma unroll
            for (int c = 0; c < 8; ++c) gp[c] += dL_dI * dI_dgeo[c];
          }
          gp[8] += pt_w * gx[k];
          gp[9] += pt_w * gy[k];
          gp[10] += pt_w * gz[k];
          gp[11] += fabsf(dL_dalpha * alpha);
        }
        // One warp reduction for both pixels' gradients of this record.
        const uint32_t act_mask = __ballot_sync(0xffffffffu, contrib);
        if (act_mask == 0u) continue;
        Acc::add(s_grad, warp, j, gp, lane, act_mask, contrib, in.atomic_lanes);
        wrote |= 1u << (j & 31);
      }
      Acc::mark(s_hit, warp, g, wrote, lane);
    }
    __syncthreads();
    // Flush this batch's accumulators: one set of vector reductions per (voxel, tile).
    for (int t = tid; t < n_here; t += CFG::NT) {
      float acc[12];
      if (!Acc::gather(s_grad, s_hit, t, acc)) continue;
      float gsum = 0.f;
#pragma unroll
      for (int c = 0; c < 12; ++c) gsum += fabsf(acc[c]);
      if (gsum != 0.f) {
        const uint32_t vid = (uint32_t)__float_as_int(s.corner[t].w);
        flush_density<GRID>(out, vid, acc, true);
        atomicAdd(reinterpret_cast<float4*>(out.dL_drgbs) + vid, make_float4(acc[8], acc[9], acc[10], acc[11]));
      }
    }
  }
}

}  // namespace svr
