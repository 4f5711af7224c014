// Per-tile compositing shared by the forward and backward kernels.
//
// A CTA of TS*TS threads owns one TSxTS pixel tile (16x16 on the plain path,
// as the reference); each warp owns an 8x4 micro-tile (forward.cu:77-92).
// Voxel instances of the tile's sorted list are staged into shared memory in
// batches of SB records (structure of arrays, vector loads where the layout
// allows), then every warp builds a
// ballot mask of the staged records whose packed bbox overlaps its 8x4
// micro-tile and whose camera quadrant matches a ray quadrant present in the
// warp.  Lanes walk only those records, in list order, so every pixel sees
// exactly the records the reference's per-pixel loop would accept
// (forward.cu:182-200), in the same order, with the same arithmetic.
#pragma once

#include <cuda_bf16.h>

#include "svr_common.cuh"
#include "svr_views.cuh"

namespace svr {

// Tile geometry and staging depth of a compositing kernel: TS x TS pixel
// tiles (TS = 8, 16 or 32), one thread per pixel, warps laid out row-major as
// 8x4 micro-tiles, SB records staged per round.
template <int TS_, int SB_>
struct TileCfg {
  static constexpr int TS = TS_;
  static constexpr int NT = TS * TS;      // threads per CTA
  static constexpr int NW = NT / 32;      // warps per CTA
  static constexpr int MX = TS / 8;       // micro-tiles per tile row
  static constexpr int SB = SB_;          // records staged per round
  static constexpr int GROUPS = SB / 32;  // 32-record ballot groups per round
  static_assert(TS == 8 || TS == 16 || TS == 32, "tile size");
  static_assert(SB % 32 == 0 && SB >= 32, "staging depth");
};
// The plain path keeps the reference's 16x16 tile lists (config.h:14-15)
// and composites each with four 8x8 CTAs that share the list.
using PlainTile = TileCfg<8, 64>;
constexpr int kPlainSub = 4;  // 8x8 CTAs per 16x16 list

// Resident CTAs per SM the compositing kernels are register-bounded for at
// 256 threads (64 registers each); other CTA sizes keep the same threads per
// SM.  Chosen by measurement on the c4 step at 8x8 tiles: forward at 3 / 4 /
// 5 / 6 gave 15.0 / 13.9 / 14.4 / 14.9 ms, backward at 3 / 4 / 5 gave
// 31.2 / 29.0 / 41.6 ms.
constexpr int kFwdMinBlocks = 4;
constexpr int kBwdMinBlocks = 4;
template <class CFG>
constexpr int fwd_min_blocks() { return CFG::NT >= 1024 ? 1 : kFwdMinBlocks * 256 / CFG::NT; }
template <class CFG>
constexpr int bwd_min_blocks() { return CFG::NT >= 1024 ? 1 : kBwdMinBlocks * 256 / CFG::NT; }
// Backward with the distortion terms: its extra per-pixel state spills at the
// 64-register budget (44-64 bytes), so those variants run one CTA fewer per
// 256 threads (85 registers at 64-thread CTAs).
template <class CFG, bool DIST>
constexpr int bwd_min_blocks_for() {
  return (DIST && CFG::NT < 1024) ? (kBwdMinBlocks - 1) * 256 / CFG::NT : bwd_min_blocks<CFG>();
}

// Pixel of thread `tid` inside its tile: warp w owns micro-tile
// (w % MX, w / MX) of 8x4 pixels, lanes row-major inside it.
template <class CFG>
__device__ __forceinline__ void tile_pixel_of(int tid, int& lx, int& ly) {
  const int warp = tid >> 5, lane = tid & 31;
  lx = (warp % CFG::MX) * 8 + (lane & 7);
  ly = (warp / CFG::MX) * 4 + (lane >> 3);
}

// Voxel attributes of one view as the kernels read them.
struct VoxelArrays {
  const uint2* bboxes;        // [P] packed pixel bbox (this view)
  const float* centers;       // [P,3]
  const float* lengths;       // [P]
  const float* geos;          // [P,8] fp32, or nullptr when geos_bf16 is set
  const __nv_bfloat16* geos_bf16;  // [P,8] bf16 storage
  const float* rgbs;          // [P,3] (this view)
  // Grid-point densities (batched grid entry points): when key is set, corner
  // c of voxel v is grid[key[8 v + c]] (fp32 grid, or grid_bf16), read while
  // staging the record, and geos / geos_bf16 are unused.
  const int64_t* key = nullptr;
  const float* grid = nullptr;
  const __nv_bfloat16* grid_bf16 = nullptr;
};

// One staged record.  Besides the raw attributes it holds the per-record
// terms of the slab test and of the sample position, computed once here
// instead of once per pixel: (c - o) -/+ l/2, c - l/2 and 1/l.  Each is the
// same IEEE operation on the same operands as in the per-pixel form, so the
// per-pixel results are unchanged bit for bit.
template <int SB>
struct StageSmem {
  uint4 box[SB];          // xmin, xmax - xmin, ymin, (ymax - ymin) | quadrant << 16
  float4 slab_lo[SB];     // (c - o) - l/2 (xyz), 1/l (w)
  float4 slab_hi[SB];     // (c - o) + l/2 (xyz), l (w)
  float4 corner[SB];      // c - l/2 (xyz), voxel id as int bits (w)
  float4 geo[SB][2];      // 8 corner densities
  float4 rgb[SB];         // rgb (xyz)
};

// MAYBE_GRID = false compiles the grid-point read out (kernels instantiated
// apart for the per-voxel densities).
template <int SB, bool MAYBE_GRID = true>
__device__ __forceinline__ void stage_record(StageSmem<SB>& s, int slot, uint32_t val, const VoxelArrays& va,
                                             float ox, float oy, float oz) {
  const uint32_t vid = val_vox_id(val);
  const uint2 bb = va.bboxes[vid];
  s.box[slot] = make_uint4(bb_xmin(bb), bb_xmax(bb) - bb_xmin(bb), bb_ymin(bb),
                           (bb_ymax(bb) - bb_ymin(bb)) | (val_quadrant(val) << 16));
  const float* c = va.centers + 3 * (size_t)vid;
  const float cx = c[0], cy = c[1], cz = c[2], len = va.lengths[vid];
  const float rad = 0.5f * len;
  const float dx = cx - ox, dy = cy - oy, dz = cz - oz;
  s.slab_lo[slot] = make_float4(dx - rad, dy - rad, dz - rad, 1.f / len);
  s.slab_hi[slot] = make_float4(dx + rad, dy + rad, dz + rad, len);
  s.corner[slot] = make_float4(cx - 0.5f * len, cy - 0.5f * len, cz - 0.5f * len, __int_as_float((int)vid));
  if (MAYBE_GRID && va.key) {
    const int64_t* k = va.key + 8 * (size_t)vid;
    float g[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) g[c] = va.grid_bf16 ? __bfloat162float(va.grid_bf16[k[c]]) : va.grid[k[c]];
    s.geo[slot][0] = make_float4(g[0], g[1], g[2], g[3]);
    s.geo[slot][1] = make_float4(g[4], g[5], g[6], g[7]);
  } else if (va.geos_bf16) {
    const uint4 raw = *reinterpret_cast<const uint4*>(va.geos_bf16 + 8 * (size_t)vid);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&raw);
    const float2 g0 = __bfloat1622float2(h[0]), g1 = __bfloat1622float2(h[1]);
    const float2 g2 = __bfloat1622float2(h[2]), g3 = __bfloat1622float2(h[3]);
    s.geo[slot][0] = make_float4(g0.x, g0.y, g1.x, g1.y);
    s.geo[slot][1] = make_float4(g2.x, g2.y, g3.x, g3.y);
  } else {
    const float4* g = reinterpret_cast<const float4*>(va.geos + 8 * (size_t)vid);
    s.geo[slot][0] = g[0];
    s.geo[slot][1] = g[1];
  }
  const float* rgb = va.rgbs + 3 * (size_t)vid;
  s.rgb[slot] = make_float4(rgb[0], rgb[1], rgb[2], 0.f);
}

// Slab test from the staged per-record terms (auxiliary.h:240-253).
__device__ __forceinline__ float2 staged_ray_box(const float4& lo, const float4& hi, const PixelRay& r) {
  const float ax = lo.x * r.ix, ay = lo.y * r.iy, az = lo.z * r.iz;
  const float bx = hi.x * r.ix, by = hi.y * r.iy, bz = hi.z * r.iz;
  const float nx = fminf(ax, bx), ny = fminf(ay, by), nz = fminf(az, bz);
  const float fx = fmaxf(ax, bx), fy = fmaxf(ay, by), fz = fmaxf(az, bz);
  return make_float2(fmaxf(fmaxf(nx, ny), nz), fminf(fminf(fx, fy), fz));
}

// Does staged record `slot` possibly touch a pixel of this warp's 8x4
// micro-tile with a matching ray quadrant?
template <int SB>
__device__ __forceinline__ bool record_hits_warp(const StageSmem<SB>& s, int slot, uint32_t wx0, uint32_t wy0,
                                                 uint32_t quad_mask) {
  const uint4 b = s.box[slot];
  return b.x <= wx0 + 7u && b.x + b.y >= wx0 && b.z <= wy0 + 3u && b.z + (b.w & 0xFFFFu) >= wy0 &&
         ((quad_mask >> (b.w >> 16)) & 1u);
}

// 32x32 bit matrix held one row per lane (bit l of lane j's word = entry
// (j, l)) to its transpose: lane l returns the column l as a word, bit j =
// entry (j, l).  Five exchanges swapping off-diagonal blocks of 16, 8, 4, 2
// and 1 columns.
__device__ __forceinline__ uint32_t warp_transpose_bits(uint32_t v, uint32_t lane) {
  const uint32_t keep[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const int d = 16 >> k;
    const uint32_t x = __shfl_xor_sync(0xffffffffu, v, d);
    const uint32_t m = keep[k];
    v = (lane & (uint32_t)d) ? ((v & ~m) | ((x >> d) & m)) : ((v & m) | ((x & m) << d));
  }
  return v;
}

// Pixels of the 8x4 block with corner (bx0, by0) that staged box b covers, as
// a 32-bit lane mask (lane = row * 8 + column; byte r = row r): the
// record_hits_pixel bbox test for 32 pixels at once.  0 when disjoint.
__device__ __forceinline__ uint32_t block_cover_mask(const uint4& b, uint32_t bx0, uint32_t by0) {
  const uint32_t x1 = b.x + b.y, y1 = b.z + (b.w & 0xFFFFu);
  if (b.x > bx0 + 7u || x1 < bx0 || b.z > by0 + 3u || y1 < by0) return 0u;
  const uint32_t cx0 = max(b.x, bx0) - bx0, cx1 = min(x1, bx0 + 7u) - bx0;
  const uint32_t ry0 = max(b.z, by0) - by0, ry1 = min(y1, by0 + 3u) - by0;
  const uint32_t cols = (0xFFu >> (7u - cx1)) & (0xFFu << cx0);
  const uint32_t rows = (0x01010101u >> (8u * (3u - ry1))) & (0x01010101u << (8u * ry0));
  return cols * rows;
}

// The reference's per-pixel test: pixel inside the packed bbox and ray
// quadrant equal to the instance's (forward.cu:186), as two unsigned range
// checks on the staged (min, extent) form.
template <int SB>
__device__ __forceinline__ bool record_hits_pixel(const StageSmem<SB>& s, int j, uint32_t px, uint32_t py,
                                                  uint32_t quad) {
  const uint4 b = s.box[j];
  return (px - b.x) <= b.y && (py - b.z) <= (b.w & 0xFFFFu) && (b.w >> 16) == quad;
}

template <int SB>
__device__ __forceinline__ void load_geo(const StageSmem<SB>& s, int j, float g[8]) {
  const float4 a = s.geo[j][0], b = s.geo[j][1];
  g[0] = a.x; g[1] = a.y; g[2] = a.z; g[3] = a.w;
  g[4] = b.x; g[5] = b.y; g[6] = b.z; g[7] = b.w;
}

// Linear-gradient "normal" of the trilinear field (forward.cu:301-310).
__device__ __forceinline__ void field_normal(const float g[8], float& nx, float& ny, float& nz) {
  nx = ((g[4] + g[5] + g[6] + g[7]) - (g[0] + g[1] + g[2] + g[3]));
  ny = ((g[2] + g[3] + g[6] + g[7]) - (g[0] + g[1] + g[4] + g[5]));
  nz = ((g[1] + g[3] + g[5] + g[7]) - (g[0] + g[2] + g[4] + g[6]));
}

}  // namespace svr
