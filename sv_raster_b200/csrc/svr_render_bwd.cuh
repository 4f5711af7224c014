// Backward compositing of one tile: walks the tile's list back to
// front from tile_last, recovers transmittance by division and accumulates
// per-voxel gradients.
//
// Per-pixel arithmetic mirrors BACKWARD::renderCUDA (backward.cu:35-530):
// contributor skip (:246-248), recomputed quadrature with dI/dgeo
// (:295-323), T recovery (:333), colour / distortion / normal / depth /
// ascending / colour-concentration terms (:344-510) and the 12-float
// gradient pack (:515-522).  The reference issues 12 global atomics per
// contributing (pixel, voxel); here each warp reduces its lanes' gradients
// with shuffles into a shared-memory accumulator per staged record
// (GradAcc), and each record is flushed once per tile (16-byte vector
// reductions where the gradient rows are aligned).
#pragma once

#include "svr_render.cuh"

namespace svr {

struct BwdTileIn {
  const float* T;          // [H*W] final transmittance from the forward
  const uint32_t* n_contrib;
  const float* dL_dcolor;  // [3,H,W]
  const float* dL_ddepth;  // [3,H,W] or nullptr
  const float* dL_dnormal; // [3,H,W] or nullptr
  const float* dL_dT;      // [H*W]
  const float* gt_color;   // [3,H,W] or nullptr
  const float* out_depth;  // [3,H,W] or nullptr (distortion prefix sums)
  float lambda_R_concen, lambda_ascending, lambda_dist;
  // A record's gradients from at most this many lanes go straight into its
  // shared accumulator with atomics; more lanes use the warp reduce-scatter.
  int atomic_lanes;
};

struct BwdTileOut {
  float* dL_dgeos;   // [P,8]
  float* dL_drgbs;   // [P,3] (this view), or [P,4] with RGB4 (xyz = dL/drgb, w = subdivision priority)
  float* subdiv;     // [P] (unused with RGB4)
  uint32_t* err;     // device error word
  int geo_vec4;      // dL_dgeos is 16-byte aligned: flush its rows with vector reductions
  // Grid-point densities: when key is set, a record's 8 corner gradients are
  // added into grid_grad[key[8 v + c]] instead of a dL_dgeos row.
  const int64_t* key = nullptr;
  float* grid_grad = nullptr;
};

// Density part of one record's flush: its 8 corner gradients into the
// voxel's dL_dgeos row (two 16-byte reductions where the rows are aligned),
// or into the grid points its corners index.
template <bool MAYBE_GRID = true>
__device__ __forceinline__ void flush_density(const BwdTileOut& out, uint32_t vid, const float acc[12], bool vec4) {
  if (MAYBE_GRID && out.key) {
    const int64_t* k = out.key + 8 * (size_t)vid;
#pragma unroll
    for (int c = 0; c < 8; ++c) atomicAdd(out.grid_grad + k[c], acc[c]);
    return;
  }
  float* g = out.dL_dgeos + 8 * (size_t)vid;
  if (vec4) {
    atomicAdd(reinterpret_cast<float4*>(g), make_float4(acc[0], acc[1], acc[2], acc[3]));
    atomicAdd(reinterpret_cast<float4*>(g) + 1, make_float4(acc[4], acc[5], acc[6], acc[7]));
  } else {
#pragma unroll
    for (int c = 0; c < 8; ++c) atomicAdd(g + c, acc[c]);
  }
}

constexpr int kGradStride = 13;  // 12 gradient floats + 1 pad (bank spread)

__device__ __forceinline__ float warp_sum(float x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Reduce-scatter of 12 per-lane values over the warp in 13 shuffles: halve
// 12 -> 6 (xor 16) -> 3 (xor 8), pad the 3 to 4 and halve 4 -> 2 (xor 4)
// -> 1 (xor 2), then add the pair (xor 1).  Lane l ends holding in v[0] the
// warp total of slot 6*b4 + 3*b3 + 2*b2 + b1 (b_i = bit i of l) when
// 2*b2 + b1 < 3; returns that slot for the even lane that should publish it
// (-1 otherwise or for the padding slot).  Every slot 0-11 is published by
// exactly one lane.
__device__ __forceinline__ int warp_reduce_scatter12(float v[12], int lane) {
  // step 1 (xor 16): keep slots 0-5 (bit 4 clear) or 6-11 (bit 4 set)
  float a[6];
  const bool hi16 = lane & 16;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const float send = hi16 ? v[k] : v[k + 6];
    const float keep = hi16 ? v[k + 6] : v[k];
    a[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  // step 2 (xor 8): keep 3 of 6
  float b[3];
  const bool hi8 = lane & 8;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float send = hi8 ? a[k] : a[k + 3];
    const float keep = hi8 ? a[k + 3] : a[k];
    b[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  // step 3 (xor 4): the 3 padded to 4, keep 2 (bit 2 set: slot 2 and the pad)
  const bool hi4 = lane & 4;
  const float c0 = (hi4 ? b[2] : b[0]) + __shfl_xor_sync(0xffffffffu, hi4 ? b[0] : b[2], 4);
  const float c1 = (hi4 ? 0.f : b[1]) + __shfl_xor_sync(0xffffffffu, hi4 ? b[1] : 0.f, 4);
  // step 4 (xor 2): keep 1 of 2
  const bool hi2 = lane & 2;
  float d = (hi2 ? c1 : c0) + __shfl_xor_sync(0xffffffffu, hi2 ? c0 : c1, 2);
  // step 5 (xor 1): full sum on both lanes of the pair
  d += __shfl_xor_sync(0xffffffffu, d, 1);
  v[0] = d;
  const int local = (hi4 ? 2 : 0) + (hi2 ? 1 : 0);
  return ((lane & 1) == 0 && local < 3) ? (hi16 ? 6 : 0) + (hi8 ? 3 : 0) + local : -1;
}

// FAST selects the arithmetic of the per-(pixel, voxel) loop (exp_f, div_f in
// svr_common.cuh); RGB4 the [P,4] colour-gradient layout whose rows, like the
// density rows, are flushed with one 16-byte vector reduction each.
// Per-record gradient accumulators of one staging round.  With at most two
// warps per CTA and 32 records staged per round, each warp owns a slot per
// staged record: a warp visits a record at most once per round, so the
// record's warp total is stored with plain stores, a bitmask per 32-record
// group marks the slots written this round, and the flush adds the (at most
// two) slots -- no shared-memory atomics and no zeroing.  Other
// configurations share one slot per record and add into it with
// shared-memory atomics (per-warp slots for 64 records would cost the 64-
// thread CTAs their 16th resident CTA per SM: measured slower).
//
// A record reached by few lanes (2 to kFewLanes, a third of the records a
// warp contributes to at 1080p over the c4 scene) is summed by transposing
// through a small per-warp area instead of the 13-shuffle reduce-scatter:
// each contributing lane stores its 12 values as one row, then lanes 0-11
// each add one column over the rows.
template <class CFG>
struct GradAcc {
  static constexpr bool kPerWarp = CFG::NW <= 2 && CFG::SB <= 32;
  static constexpr int kStride = kPerWarp ? 12 : kGradStride;  // 48-byte rows: 16-byte vector access
  static constexpr int kFewLanes = 8;
  static constexpr int kSlots = (kPerWarp ? CFG::NW : 1) * CFG::SB * kStride;
  // accumulators, then the transposition rows (16-byte aligned)
  static constexpr int kRowsAt = (kSlots + 3) / 4 * 4;
  static constexpr int kFloats = kRowsAt + CFG::NW * kFewLanes * 12;
  static constexpr int kWords = kPerWarp ? CFG::NW * CFG::GROUPS : 1;

  __device__ static void init(float* s_grad, int tid) {
    if (!kPerWarp)
      for (int i = tid; i < CFG::SB * kStride; i += CFG::NT) s_grad[i] = 0.f;
  }

  // The warp's gradients of staged record j (gp: this lane's 12 values,
  // meaningful where `contrib`; act_mask: the contributing lanes).
  __device__ static void add(float* s_grad, int warp, int j, float gp[12], int lane, uint32_t act_mask,
                             bool contrib, int atomic_lanes) {
    const int k = __popc(act_mask);
    float* acc = s_grad + ((kPerWarp ? warp * CFG::SB : 0) + j) * kStride;
    if (kPerWarp ? k == 1 : k <= atomic_lanes) {
      if (contrib) {  // one (or, shared slots, a few) lane(s): their values go straight in
        if (kPerWarp) store_row(acc, gp);
        else
#pragma unroll
          for (int c = 0; c < 12; ++c) atomicAdd(acc + c, gp[c]);
      }
    } else if (k <= kFewLanes) {
      float* rows = s_grad + kRowsAt + warp * kFewLanes * 12;
      if (contrib) store_row(rows + 12 * __popc(act_mask & ((1u << lane) - 1u)), gp);
      __syncwarp();
      if (lane < 12) {
        float sum = rows[lane];
        for (int r = 1; r < k; ++r) sum += rows[12 * r + lane];
        if (kPerWarp) acc[lane] = sum;
        else atomicAdd(acc + lane, sum);
      }
      __syncwarp();  // the rows are reused by the warp's next record
    } else {
      if (!contrib) {
#pragma unroll
        for (int c = 0; c < 12; ++c) gp[c] = 0.f;
      }
      const int slot = warp_reduce_scatter12(gp, lane);
      if (slot >= 0) {
        if (kPerWarp) acc[slot] = gp[0];
        else atomicAdd(acc + slot, gp[0]);
      }
    }
  }

  __device__ static void store_row(float* row, const float gp[12]) {
    float4* a4 = reinterpret_cast<float4*>(row);
    a4[0] = make_float4(gp[0], gp[1], gp[2], gp[3]);
    a4[1] = make_float4(gp[4], gp[5], gp[6], gp[7]);
    a4[2] = make_float4(gp[8], gp[9], gp[10], gp[11]);
  }

  // End of group g of a warp's hit loop: `wrote` marks the records it stored.
  __device__ static void mark(uint32_t* s_hit, int warp, int g, uint32_t wrote, int lane) {
    if (kPerWarp && lane == 0) s_hit[warp * CFG::GROUPS + g] = wrote;
  }

  // Record t's total over the CTA this round; false when no warp wrote it.
  __device__ static bool gather(float* s_grad, const uint32_t* s_hit, int t, float a[12]) {
    if (kPerWarp) {
      bool any = false;
#pragma unroll
      for (int c = 0; c < 12; ++c) a[c] = 0.f;
#pragma unroll
      for (int w = 0; w < CFG::NW; ++w) {
        if (!((s_hit[w * CFG::GROUPS + (t >> 5)] >> (t & 31)) & 1u)) continue;
        any = true;
        const float4* a4 = reinterpret_cast<const float4*>(s_grad + (w * CFG::SB + t) * kStride);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const float4 v = a4[q];
          a[4 * q] += v.x; a[4 * q + 1] += v.y; a[4 * q + 2] += v.z; a[4 * q + 3] += v.w;
        }
      }
      return any;
    }
    float* acc = s_grad + t * kStride;
#pragma unroll
    for (int c = 0; c < 12; ++c) {
      a[c] = acc[c];
      acc[c] = 0.f;
    }
    return true;
  }
};

// Per-pixel state of the backward walk (the pixel's upstream gradients, its
// transmittance being recovered record by record, and the running sums).
struct BwdPix {
  float T, last_dL_dT;
  float gx, gy, gz, dL_dD, dNx, dNy, dNz, gtx, gty, gtz;
  float weight_R, weight_asc, weight_dist;
  float prefix_wm, suffix_wm, prefix_w, suffix_w;
};

template <bool DEPTH, bool DIST, bool NORMAL>
__device__ __forceinline__ BwdPix bwd_pixel_init(const ViewParams& vp, const BwdTileIn& in, const PixelRay& ray,
                                                 bool inside, uint32_t pix_id, float T_final) {
  const int W = vp.W, H = vp.H;
  const size_t HW = (size_t)H * W;
  BwdPix st;
  st.T = T_final;
  st.gx = 0.f; st.gy = 0.f; st.gz = 0.f; st.last_dL_dT = 0.f; st.dL_dD = 0.f;
  st.dNx = 0.f; st.dNy = 0.f; st.dNz = 0.f;
  if (inside) {
    st.gx = in.dL_dcolor[0 * HW + pix_id];
    st.gy = in.dL_dcolor[1 * HW + pix_id];
    st.gz = in.dL_dcolor[2 * HW + pix_id];
    const float dT = in.dL_dT[pix_id];
    st.last_dL_dT = dT + vp.bg * (st.gx + st.gy + st.gz);
    if (DEPTH) st.dL_dD = in.dL_ddepth[pix_id] * ray.rd_norm_inv;
    if (NORMAL) {
      st.dNx = in.dL_dnormal[0 * HW + pix_id];
      st.dNy = in.dL_dnormal[1 * HW + pix_id];
      st.dNz = in.dL_dnormal[2 * HW + pix_id];
    }
  }
  const float WH_inv = 1.f / ((float)(W * H));
  st.weight_R = in.lambda_R_concen * WH_inv;
  st.weight_asc = in.lambda_ascending * WH_inv;
  st.gtx = 0.f; st.gty = 0.f; st.gtz = 0.f;
  if (in.lambda_R_concen > 0 && inside) {
    st.gtx = in.gt_color[0 * HW + pix_id];
    st.gty = in.gt_color[1 * HW + pix_id];
    st.gtz = in.gt_color[2 * HW + pix_id];
  }
  st.weight_dist = in.lambda_dist * WH_inv;
  st.prefix_wm = 0.f; st.suffix_wm = 0.f; st.prefix_w = 0.f; st.suffix_w = 0.f;
  if (DIST && inside) {
    st.prefix_wm = in.out_depth[HW + pix_id];
    st.prefix_w = 1.f - T_final;
  }
  return st;
}

// One (pixel, staged record j) step of the backward walk, for a pixel inside
// the record's bbox with a matching quadrant: slab test, recomputed
// quadrature, T recovery and the 12 gradient values (8 density corners, 3
// colour, 1 subdivision priority) in gp.  Returns whether the record
// contributes (gp is left unset otherwise).
template <int SB, int NS, bool DEPTH, bool DIST, bool NORMAL, bool FAST>
__device__ __forceinline__ bool bwd_pixel_record(const StageSmem<SB>& s, int j, const PixelRay& ray,
                                                 const BwdTileIn& in, BwdPix& st, float gp[12]) {
  float& T = st.T;
  float& last_dL_dT = st.last_dL_dT;
  float& prefix_wm = st.prefix_wm;
  float& suffix_wm = st.suffix_wm;
  float& prefix_w = st.prefix_w;
  float& suffix_w = st.suffix_w;
  const float gx = st.gx, gy = st.gy, gz = st.gz, dL_dD = st.dL_dD;
  const float dNx = st.dNx, dNy = st.dNy, dNz = st.dNz, gtx = st.gtx, gty = st.gty, gtz = st.gtz;
  const float weight_R = st.weight_R, weight_asc = st.weight_asc, weight_dist = st.weight_dist;
  (void)dL_dD; (void)dNx; (void)dNy; (void)dNz; (void)weight_dist;
  (void)prefix_wm; (void)suffix_wm; (void)prefix_w; (void)suffix_w;
  bool contrib = false;
  // Fast arithmetic, one sample, no depth terms: keep the trilinear weights
  // and scale them once by dL/dI * d(density)/d(sample) (8 multiplies fewer
  // than forming dI/dgeo first; a different rounding order).
  constexpr bool kFoldScale = FAST && NS == 1 && !DEPTH;
  const float4 slo = s.slab_lo[j], shi = s.slab_hi[j];
  const float2 ab = staged_ray_box(slo, shi, ray);
  const float a = ab.x, b = ab.y;
  if (!(a > b)) {
    float geo[8];
    load_geo(s, j, geo);
    float dgeo[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) dgeo[c] = 0.f;
    float vol_int = 0.f;
    float dI_dgeo[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) dI_dgeo[c] = 0.f;
    float each_dI[NS][8];
    float w[8];
    float local_alpha[NS];
    const float vox_l_inv = slo.w;
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
      float act, act_grad;
      density_act_and_grad_f<FAST>(d, act, act_grad);
      const float lvi = kStepScale * step_sz * act;
      vol_int += lvi;
      if (DEPTH && NS > 1) local_alpha[k] = fminf(kMaxAlpha, 1.f - exp_f<FAST>(-lvi));
      const float dd_dd = kStepScale * step_sz * act_grad;
      if (kFoldScale) {
        dI_dgeo[0] = dd_dd;  // the weights stay in w: dL/dgeo = (dL/dI * dd_dd) * w below
      } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float tmp = dd_dd * w[c];
          dI_dgeo[c] += tmp;
          if (DEPTH && NS > 1) each_dI[k][c] = tmp;
        }
      }
      qx = qx + qsx; qy = qy + qsy; qz = qz + qsz;
    }
    const float exp_neg = exp_f<FAST>(-vol_int);
    const float alpha = fminf(kMaxAlpha, 1.f - exp_neg);
    if (!(alpha < kMinAlpha)) {
      contrib = true;
      T = div_f<FAST>(T, 1.f - alpha);
      const float pt_w = alpha * T;
      const float4 rgbv = s.rgb[j];
      float dL_dpt_w = gx * rgbv.x + gy * rgbv.y + gz * rgbv.z;
      if (DIST) {
        const float adist = contract_depth(a), bdist = contract_depth(b);
        const float now_m = 0.5f * (adist + bdist);
        const float now_wm = now_m * pt_w;
        prefix_wm -= now_wm;
        prefix_w -= pt_w;
        const float uni = 0.6666666f * pt_w * (bdist - adist);
        const float bi = 2.f * (now_m * (prefix_w - suffix_w) - (prefix_wm - suffix_wm));
        dL_dpt_w += weight_dist * (uni + bi);
        suffix_wm += now_wm;
        suffix_w += pt_w;
      }
      if (NORMAL) {
        float nx, ny, nz;
        field_normal(geo, nx, ny, nz);
        const float rl = safe_rnorm3(nx, ny, nz);
        const float sx = rl * nx, sy = rl * ny, sz = rl * nz;
        dL_dpt_w += dNx * sx + dNy * sy + dNz * sz;
        const float dsx = pt_w * dNx, dsy = pt_w * dNy, dsz = pt_w * dNz;
        const float dot_ = dsx * nx + dsy * ny + dsz * nz;
        const float lnx = rl * (dsx - dot_ * rl * sx);
        const float lny = rl * (dsy - dot_ * rl * sy);
        const float lnz = rl * (dsz - dot_ * rl * sz);
        dgeo[0] += -lnx - lny - lnz;
        dgeo[1] += -lnx - lny + lnz;
        dgeo[2] += -lnx + lny - lnz;
        dgeo[3] += -lnx + lny + lnz;
        dgeo[4] += +lnx - lny - lnz;
        dgeo[5] += +lnx - lny + lnz;
        dgeo[6] += +lnx + lny - lnz;
        dgeo[7] += +lnx + lny + lnz;
      }
      const float dL_dalpha = T * (dL_dpt_w - last_dL_dT);
      last_dL_dT += alpha * (dL_dpt_w - last_dL_dT);
      const float dL_dI = dL_dalpha * exp_neg;
      if (kFoldScale) {
        const float sI = dL_dI * dI_dgeo[0];
#pragma unroll
        for (int c = 0; c < 8; ++c) dgeo[c] += sI * w[c];
      } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) dgeo[c] += dL_dI * dI_dgeo[c];
      }
      if (DEPTH) {
        float dval;
        float dI[NS];
        if (NS == 3) {
          const float ss = 0.3333333f * (b - a);
          const float a0 = local_alpha[0], a1 = local_alpha[NS > 1 ? 1 : 0], a2 = local_alpha[NS > 2 ? 2 : 0];
          const float t0_ = a + 0.5f * ss, t1_ = a + 1.5f * ss, t2_ = a + 2.5f * ss;
          dval = a0 * t0_ + (1.f - a0) * a1 * t1_ + (1.f - a0) * (1.f - a1) * a2 * t2_;
          dI[0] = dL_dD * T * (t0_ + a1 * a2 * t2_ - a1 * t1_ - a2 * t2_) * (1.f - a0);
          dI[NS > 1 ? 1 : 0] = dL_dD * T * (t1_ + a0 * a2 * t2_ - a0 * t1_ - a2 * t2_) * (1.f - a1);
          dI[NS > 2 ? 2 : 0] = dL_dD * T * (t2_ + a0 * a1 * t2_ - a0 * t2_ - a1 * t2_) * (1.f - a2);
        } else if (NS == 2) {
          const float ss = 0.5f * (b - a);
          const float a0 = local_alpha[0], a1 = local_alpha[NS > 1 ? 1 : 0];
          const float t0_ = a + 0.5f * ss, t1_ = a + 1.5f * ss;
          dval = a0 * t0_ + (1.f - a0) * a1 * t1_;
          dI[0] = dL_dD * T * (t0_ - a1 * t1_) * (1.f - a0);
          dI[NS > 1 ? 1 : 0] = dL_dD * T * (t1_ - a0 * t1_) * (1.f - a1);
        } else {
          const float t0_ = 0.5f * (a + b);
          dval = alpha * t0_;
          dI[0] = dL_dD * T * t0_ * (1.f - alpha);
        }
        last_dL_dT += dL_dD * dval;
        if (NS == 3) {
#pragma unroll
          for (int c = 0; c < 8; ++c)
            dgeo[c] += dI[0] * each_dI[0][c] + dI[NS > 1 ? 1 : 0] * each_dI[NS > 1 ? 1 : 0][c] +
                       dI[NS > 2 ? 2 : 0] * each_dI[NS > 2 ? 2 : 0][c];
        } else if (NS == 2) {
#pragma unroll
          for (int c = 0; c < 8; ++c)
            dgeo[c] += dI[0] * each_dI[0][c] + dI[NS > 1 ? 1 : 0] * each_dI[NS > 1 ? 1 : 0][c];
        } else {
#pragma unroll
          for (int c = 0; c < 8; ++c) dgeo[c] += dI[0] * dI_dgeo[c];
        }
      }
      if (in.lambda_ascending > 0) {
        const float lo_x = cr.x, lo_y = cr.y, lo_z = cr.z;
        const float pax = ray.ox + a * ray.dx, pay = ray.oy + a * ray.dy, paz = ray.oz + a * ray.dz;
        const float pbx = ray.ox + b * ray.dx, pby = ray.oy + b * ray.dy, pbz = ray.oz + b * ray.dz;
        float wa[8], wb[8];
        trilinear_weights((pax - lo_x) * vox_l_inv, (pay - lo_y) * vox_l_inv, (paz - lo_z) * vox_l_inv, wa);
        trilinear_weights((pbx - lo_x) * vox_l_inv, (pby - lo_y) * vox_l_inv, (pbz - lo_z) * vox_l_inv, wb);
        float d_a = 0.f, d_b = 0.f;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          d_a += geo[c] * wa[c];
          d_b += geo[c] * wb[c];
        }
        const float reg_w = weight_asc * pt_w * static_cast<float>(d_a > d_b);
#pragma unroll
        for (int c = 0; c < 8; ++c) dgeo[c] += reg_w * (wa[c] - wb[c]);
      }
      float drx = pt_w * gx, dry = pt_w * gy, drz = pt_w * gz;
      if (in.lambda_R_concen > 0) {
        const float sR = weight_R * pt_w * 2.0f;
        drx += sR * (rgbv.x - gtx);
        dry += sR * (rgbv.y - gty);
        drz += sR * (rgbv.z - gtz);
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) gp[c] = dgeo[c];
      gp[8] = drx; gp[9] = dry; gp[10] = drz;
      gp[11] = fabsf(dL_dalpha * alpha);
    }
  }
  return contrib;
}

template <class CFG, int NS, bool DEPTH, bool DIST, bool NORMAL, bool FAST = false, bool RGB4 = false>
__device__ __forceinline__ void render_tile_bwd(const ViewParams& vp, const float* __restrict__ c2w_s, int tile_x,
                                                int tile_y, uint2 range_raw, uint32_t tile_last,
                                                const uint32_t* __restrict__ vals, const VoxelArrays& va,
                                                const BwdTileIn& in, const BwdTileOut& out, StageSmem<CFG::SB>& s,
                                                float* s_grad /*[GradAcc::kFloats]*/,
                                                uint32_t* s_hit /*[GradAcc::kWords]*/) {
  using Acc = GradAcc<CFG>;
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
  BwdPix st = bwd_pixel_init<DEPTH, DIST, NORMAL>(vp, in, ray, inside, pix_id, T_final);

  Acc::init(s_grad, tid);
  // Largest contributor count of this warp: records at or beyond it are skipped by every lane.
  const uint32_t warp_lc = __reduce_max_sync(0xffffffffu, last_contrib);
  const uint32_t quad_mask = __reduce_or_sync(0xffffffffu, inside ? (1u << ray.quad) : 0u);
  // Lane q holds the lanes whose pixel is in the image with ray quadrant q.
  uint32_t qlanes = 0u;
  for (uint32_t qm = quad_mask; qm; qm &= qm - 1) {
    const uint32_t q = (uint32_t)(__ffs(qm) - 1);
    const uint32_t bq = __ballot_sync(0xffffffffu, inside && ray.quad == q);
    if ((uint32_t)lane == q) qlanes = bq;
  }

  const int rounds = (todo_total + SB - 1) / SB;
  for (int r = 0; r < rounds; ++r) {
    __syncthreads();
    const int base = r * SB;                     // records [base, base+n_here) from the back
    const int n_here = min(SB, todo_total - base);
    for (int i = tid; i < n_here; i += CFG::NT)
      stage_record(s, i, vals[range.y - base - i - 1], va, ray.ox, ray.oy, ray.oz);
    __syncthreads();

    // Position (relative to range.x) of staged slot j is todo_total - base - j - 1.
    for (int g = 0; g < CFG::GROUPS && g * 32 < n_here; ++g) {
      const int slot = g * 32 + lane;
      const uint32_t pos = (uint32_t)(todo_total - base - slot - 1);
      const bool hit = slot < n_here && pos < warp_lc && record_hits_warp(s, slot, wx0, wy0, quad_mask);
      uint32_t m = __ballot_sync(0xffffffffu, hit);
      // This lane's candidate records of the group (pixel in the record's
      // bbox, matching quadrant, record within the contributor count): lane
      // j's block mask of record j, transposed across the warp.
      uint32_t covers = 0u, rec_quad = 0u;
      if (hit) {
        const uint4 b = s.box[slot];
        covers = block_cover_mask(b, wx0, wy0);
        rec_quad = b.w >> 16;
      }
      uint32_t mine = warp_transpose_bits(covers & __shfl_sync(0xffffffffu, qlanes, (int)rec_quad), (uint32_t)lane);
      {
        // slot j is in reach while todo_total - base - j - 1 < last_contrib
        const int first = todo_total - base - (int)last_contrib - g * 32;
        mine &= first <= 0 ? 0xffffffffu : (first >= 32 ? 0u : ~((1u << first) - 1u));
      }
      m &= __reduce_or_sync(0xffffffffu, mine);  // records no pixel of the warp takes
      uint32_t wrote = 0u;
      while (m) {
        const int bit = __ffs(m) - 1;
        const int j = g * 32 + bit;
        m &= m - 1;
        bool contrib = false;
        float gp[12];
        if ((mine >> bit) & 1u) contrib = bwd_pixel_record<SB, NS, DEPTH, DIST, NORMAL, FAST>(s, j, ray, in, st, gp);
        // Warp reduction of this record's gradients into its accumulator.
        const uint32_t act_mask = __ballot_sync(0xffffffffu, contrib);
        if (act_mask == 0u) continue;
        Acc::add(s_grad, warp, j, gp, lane, act_mask, contrib, in.atomic_lanes);
        wrote |= 1u << (j & 31);
      }
      Acc::mark(s_hit, warp, g, wrote, lane);
    }
    __syncthreads();
    // Flush this batch's accumulators: one set of reductions per (voxel, tile).
    for (int t = tid; t < n_here; t += CFG::NT) {
      float acc[12];
      if (!Acc::gather(s_grad, s_hit, t, acc)) continue;
      float gsum = 0.f;
#pragma unroll
      for (int c = 0; c < 12; ++c) gsum += fabsf(acc[c]);
      if (gsum != 0.f) {
        const uint32_t vid = (uint32_t)__float_as_int(s.corner[t].w);
        flush_density(out, vid, acc, RGB4 || out.geo_vec4);
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
