// Forward compositing of one tile: front-to-back alpha blending of the
// tile's sorted voxel instances with trilinear density quadrature.
//
// Per-pixel arithmetic mirrors FORWARD::renderCUDA (forward.cu:39-392):
// ray setup (:100-111), slab test (:192), n_samp midpoint quadrature
// (:228-248), alpha clamp and MIN_ALPHA skip (:251-253), colour / depth /
// distortion / normal accumulation (:256-313), early stop at T < 1e-4
// (:315-316), median-depth refinement (:328-364) and outputs (:368-391).
// Differences are in scheduling only: SoA staging, warp-ballot culling of the
// staged batch, each lane walking its own pixel's records of the batch, a
// single pass per pixel instead of the collect-then-process two-pass with a
// 256-entry local array, and a CTA reduction for tile_last.
#pragma once

#include "svr_render.cuh"

namespace svr {

struct FwdTileOut {
  uint32_t* tile_last;   // [T] of this view (indexed by the callers)
  uint32_t* n_contrib;   // [H*W] of this view
  float* color;          // [3,H,W]
  float* depth;          // [3,H,W] or nullptr
  float* normal;         // [3,H,W] or nullptr
  float* T;              // [H*W]
  float* max_w;          // [P] or nullptr
};

// (tile_x, tile_y) index CFG::TS-sized tiles; `range` is the list the tile
// walks (its own, or the list of an enclosing tile it shares with others);
// `last_slot` receives range.x + the tile's largest contributor count, with
// atomicMax when SHARED_LAST (several CTAs share one list and slot, which
// then starts at 0).
// FAST selects the arithmetic of the per-(pixel, voxel) loop (exp_f, svr_common.cuh).
template <class CFG, int NS, bool DEPTH, bool DIST, bool NORMAL, bool MAXW, bool SHARED_LAST = false, bool FAST = false>
__device__ __forceinline__ void render_tile_fwd(const ViewParams& vp, const float* __restrict__ c2w_s, int tile_x,
                                                int tile_y, uint2 range, const uint32_t* __restrict__ vals,
                                                const VoxelArrays& va, const FwdTileOut& out, uint32_t* last_slot,
                                                StageSmem<CFG::SB>& s, uint32_t* s_red /*[CFG::NW]*/) {
  constexpr int SB = CFG::SB;
  const int W = vp.W, H = vp.H;
  const int tid = threadIdx.x;
  int lx, ly;
  tile_pixel_of<CFG>(tid, lx, ly);
  const uint32_t px = tile_x * CFG::TS + lx, py = tile_y * CFG::TS + ly;
  const uint32_t pix_id = (uint32_t)W * py + px;
  const bool inside = px < (uint32_t)W && py < (uint32_t)H;
  const PixelRay ray = make_pixel_ray((float)px, (float)py, W, H, vp.tanfovx, vp.tanfovy, vp.cx, vp.cy, c2w_s);
  const int warp = tid >> 5;
  const uint32_t wx0 = tile_x * CFG::TS + (warp % CFG::MX) * 8, wy0 = tile_y * CFG::TS + (warp / CFG::MX) * 4;

  bool done = !inside;
  float T = 1.f;
  float Cx = 0.f, Cy = 0.f, Cz = 0.f;
  float Nx = 0.f, Ny = 0.f, Nz = 0.f;
  float D = 0.f, Ddist = 0.f;
  int dmed_vid = -1;
  float dmed_T = 0.f;
  uint32_t last_contrib = 0;

  const int todo_total = (int)(range.y - range.x);
  const int rounds = (todo_total + SB - 1) / SB;
  for (int r = 0; r < rounds; ++r) {
    // All pixels finished: stop (also the barrier that frees the staging buffer).
    if (__syncthreads_count(done) == CFG::NT) break;
    const int base = r * SB;
    const int n_here = min(SB, todo_total - base);
    for (int i = tid; i < n_here; i += CFG::NT)
      stage_record(s, i, vals[range.x + base + i], va, ray.ox, ray.oy, ray.oz);
    __syncthreads();

    const uint32_t quad_mask = __reduce_or_sync(0xffffffffu, done ? 0u : (1u << ray.quad));
    if (quad_mask == 0u) continue;  // whole warp finished
    // Lane q holds the mask of lanes still compositing whose ray quadrant is q.
    const uint32_t lane = tid & 31;
    uint32_t qlanes = 0u;
    for (uint32_t qm = quad_mask; qm; qm &= qm - 1) {
      const uint32_t q = (uint32_t)(__ffs(qm) - 1);
      const uint32_t b = __ballot_sync(0xffffffffu, !done && ray.quad == q);
      if (lane == q) qlanes = b;
    }
    for (int g = 0; g < CFG::GROUPS && g * 32 < n_here; ++g) {
      const int slot = g * 32 + (int)lane;
      const bool hit = slot < n_here && record_hits_warp(s, slot, wx0, wy0, quad_mask);
      // Lane j: the pixels of the warp's 8x4 block that staged record j
      // covers with a matching ray quadrant (record_hits_pixel for all 32
      // pixels at once: the bbox clipped to the block, as byte rows).
      uint32_t covers = 0u;
      uint32_t rec_quad = 0u;
      if (hit) {
        const uint4 b = s.box[slot];
        covers = block_cover_mask(b, wx0, wy0);
        rec_quad = b.w >> 16;
      }
      covers &= __shfl_sync(0xffffffffu, qlanes, (int)rec_quad);
      // This pixel's records among those (a transposition of the 32 masks):
      // each lane then walks its own list in order, so one warp iteration
      // serves a different record per lane (a warp takes as many iterations
      // as its busiest pixel has records, not one per record that touches it).
      // (qlanes was taken at the start of the round: a pixel that finished in
      // an earlier group of this round takes no more records.)
      uint32_t mine = warp_transpose_bits(covers, lane);
      if (done) mine = 0u;
      while (mine) {
        const int j = g * 32 + __ffs(mine) - 1;
        mine &= mine - 1;
        const float4 slo = s.slab_lo[j], shi = s.slab_hi[j];
        const float2 ab = staged_ray_box(slo, shi, ray);
        const float a = ab.x, b = ab.y;
        if (a > b) continue;

        float geo[8];
        load_geo(s, j, geo);
        float vol_int = 0.f;
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
          const float lvi = kStepScale * step_sz * density_act_f<FAST>(d);
          vol_int += lvi;
          if (DEPTH && NS > 1) local_alpha[k] = fminf(kMaxAlpha, 1.f - exp_f<FAST>(-lvi));
          qx = qx + qsx; qy = qy + qsy; qz = qz + qsz;
        }
        const float alpha = fminf(kMaxAlpha, 1.f - exp_f<FAST>(-vol_int));
        if (alpha < kMinAlpha) continue;

        const float pt_w = T * alpha;
        const float4 rgbv = s.rgb[j];
        const int vid = __float_as_int(cr.w);
        Cx = Cx + pt_w * rgbv.x;
        Cy = Cy + pt_w * rgbv.y;
        Cz = Cz + pt_w * rgbv.z;
        if (DEPTH) {
          float dval;
          if (NS == 3) {
            const float ss = 0.3333333f * (b - a);
            const float a0 = local_alpha[0], a1 = local_alpha[NS > 1 ? 1 : 0], a2 = local_alpha[NS > 2 ? 2 : 0];
            const float t0_ = a + 0.5f * ss, t1_ = a + 1.5f * ss, t2_ = a + 2.5f * ss;
            dval = a0 * t0_ + (1.f - a0) * a1 * t1_ + (1.f - a0) * (1.f - a1) * a2 * t2_;
          } else if (NS == 2) {
            const float ss = 0.5f * (b - a);
            const float a0 = local_alpha[0], a1 = local_alpha[NS > 1 ? 1 : 0];
            const float t0_ = a + 0.5f * ss, t1_ = a + 1.5f * ss;
            dval = a0 * t0_ + (1.f - a0) * a1 * t1_;
          } else {
            dval = alpha * 0.5f * (a + b);
          }
          D = D + T * dval;
          if (T > 0.5f) {
            dmed_vid = vid;
            dmed_T = T;
          }
        }
        if (DIST) Ddist = Ddist + pt_w * 0.5f * (contract_depth(a) + contract_depth(b));
        if (NORMAL) {
          float nx, ny, nz;
          field_normal(geo, nx, ny, nz);
          const float rl = safe_rnorm3(nx, ny, nz);
          Nx = Nx + pt_w * rl * nx;
          Ny = Ny + pt_w * rl * ny;
          Nz = Nz + pt_w * rl * nz;
        }
        T *= (1.f - alpha);
        last_contrib = (uint32_t)(base + j + 1);
        if (MAXW) atomicMax(reinterpret_cast<int*>(out.max_w) + vid, __float_as_int(pt_w));
        if (T < kEarlyStopT) {
          done = true;
          mine = 0u;
        }
      }
    }
  }

  float Dmed = 0.f;
  if (DEPTH && inside && dmed_vid != -1) {
    // Median depth refined with 16 samples inside the voxel where T crosses 0.5.
    constexpr int kMedSamples = 16;
    const float* c = va.centers + 3 * (size_t)dmed_vid;
    const float cxv = c[0], cyv = c[1], czv = c[2], lv = va.lengths[dmed_vid];
    float geo[8];
    if (va.geos_bf16) {
      for (int k = 0; k < 8; ++k) geo[k] = __bfloat162float(va.geos_bf16[8 * (size_t)dmed_vid + k]);
    } else {
      for (int k = 0; k < 8; ++k) geo[k] = va.geos[8 * (size_t)dmed_vid + k];
    }
    const float2 ab = ray_box(cxv, cyv, czv, lv, ray);
    const float a = ab.x, b = ab.y;
    const float vox_l_inv = 1.f / lv;
    const float step_sz = (b - a) * (1.f / kMedSamples);
    const float stx = step_sz * ray.dx, sty = step_sz * ray.dy, stz = step_sz * ray.dz;
    const float t0 = a + 0.5f * step_sz;
    const float ptx = ray.ox + t0 * ray.dx, pty = ray.oy + t0 * ray.dy, ptz = ray.oz + t0 * ray.dz;
    float qx = (ptx - (cxv - 0.5f * lv)) * vox_l_inv;
    float qy = (pty - (cyv - 0.5f * lv)) * vox_l_inv;
    float qz = (ptz - (czv - 0.5f * lv)) * vox_l_inv;
    const float qsx = stx * vox_l_inv, qsy = sty * vox_l_inv, qsz = stz * vox_l_inv;
    Dmed = a - 0.5f * step_sz;
    for (int k = 0; k < kMedSamples && dmed_T > 0.5f; k++) {
      Dmed += step_sz;
      float w[8];
      trilinear_weights(qx, qy, qz, w);
      float d = 0.f;
      for (int cc = 0; cc < 8; ++cc) d += geo[cc] * w[cc];
      const float vol_int = kStepScale * step_sz * density_act(d);
      dmed_T *= expf(-vol_int);
      qx = qx + qsx; qy = qy + qsy; qz = qz + qsz;
    }
  }

  const size_t HW = (size_t)H * W;
  if (inside) {
    out.n_contrib[pix_id] = last_contrib;
    out.color[0 * HW + pix_id] = Cx + T * vp.bg;
    out.color[1 * HW + pix_id] = Cy + T * vp.bg;
    out.color[2 * HW + pix_id] = Cz + T * vp.bg;
    out.T[pix_id] = T;
    if (DEPTH) {
      out.depth[pix_id] = D * ray.rd_norm_inv;
      out.depth[2 * HW + pix_id] = Dmed * ray.rd_norm_inv;
    }
    if (DIST) out.depth[HW + pix_id] = Ddist;
    if (NORMAL) {
      out.normal[0 * HW + pix_id] = Nx;
      out.normal[1 * HW + pix_id] = Ny;
      out.normal[2 * HW + pix_id] = Nz;
    }
  }
  // tile_last = range start + the largest contributor count of the tile.
  const uint32_t lc = __reduce_max_sync(0xffffffffu, inside ? last_contrib : 0u);
  if ((tid & 31) == 0) s_red[tid >> 5] = lc;
  __syncthreads();
  if (tid == 0) {
    uint32_t m = 0;
#pragma unroll
    for (int w = 0; w < CFG::NW; ++w) m = max(m, s_red[w]);
    if (SHARED_LAST) atomicMax(last_slot, range.x + m);
    else *last_slot = range.x + m;
  }
}

}  // namespace svr
