// Shared device-side definitions for the sm_100a sparse-voxel rasterizer.
//
// Numerical conventions follow the reference backend (panicPaul/sv_raster,
// backends/cuda/src/config.h:14-28 and auxiliary.h).  Every floating-point
// expression that feeds an early-termination or culling decision is written
// with the same operation order as the reference so that, compiled by nvcc
// with the same default contraction (-fmad=true, no fast-math), contributor
// counts and tile lists come out bit-identical.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "svr_status.h"

namespace svr {

// Tile geometry of the parity path (config.h:14-15).  Contributor indices and
// tile lists are only comparable with the reference at 16x16 tiles; the
// batched path may use 8x8 or 32x32 tiles (ViewParams::tile_shift).
constexpr int kTileX = 16;
constexpr int kTileY = 16;
constexpr int kTileShift = 4;

constexpr int kMaxLevels = 16;                    // config.h:16
constexpr float kMaxAlpha = 0.99999f;             // config.h:17
constexpr float kMinAlpha = 0.00001f;             // config.h:18
constexpr float kEarlyStopT = 0.0001f;            // config.h:19
constexpr float kStepScale = 100.f;               // config.h:21
constexpr int kMaxSamples = 3;                    // config.h:23
constexpr int kRankBits = 3 * kMaxLevels;         // config.h:27 (48)
constexpr int kVoxIdBits = 29;                    // auxiliary.h:50-63
// Octrees 21 levels deep (the reference's new_cuda backend, config.h:16,30):
// 63-bit Morton ranks, sorted as (tile, rank) pairs wider than 64 bits.
constexpr int kDeepLevels = 21;
constexpr int kDeepRankBits = 3 * kDeepLevels;

// Repeat a 3-bit octant code over all 16 octree levels (auxiliary.h:16-38).
__host__ __device__ constexpr uint64_t octant_repeat(uint64_t q) {
  uint64_t v = 0;
  for (int l = 0; l < kMaxLevels; ++l) v = (v << 3) | q;
  return v;
}

// Direction-dependent Morton rank: flipping every octant digit by the camera
// quadrant turns "front to back" into ascending order (auxiliary.h:40-43).
__device__ __forceinline__ uint64_t order_rank(uint64_t octpath, uint32_t q) {
  return octpath ^ octant_repeat(q);
}

__device__ __forceinline__ uint64_t make_sort_key(uint64_t tile, uint64_t rank) {
  return (tile << kRankBits) | rank;
}

__device__ __forceinline__ uint32_t make_sort_val(uint32_t vid, uint32_t q) {
  return (q << kVoxIdBits) | vid;
}

__device__ __forceinline__ uint32_t val_vox_id(uint32_t v) { return v & ((1u << kVoxIdBits) - 1u); }
__device__ __forceinline__ uint32_t val_quadrant(uint32_t v) { return v >> kVoxIdBits; }

// Packed pixel bbox: .x = xmin<<16 | ymin, .y = xmax<<16 | ymax (preprocess.cu:110-113).
__device__ __forceinline__ uint32_t bb_xmin(uint2 b) { return b.x >> 16; }
__device__ __forceinline__ uint32_t bb_ymin(uint2 b) { return b.x & 0xFFFFu; }
__device__ __forceinline__ uint32_t bb_xmax(uint2 b) { return b.y >> 16; }
__device__ __forceinline__ uint32_t bb_ymax(uint2 b) { return b.y & 0xFFFFu; }

// Tile rectangle covered by a packed bbox, clamped to the tile grid
// (auxiliary.h:86-100), for square tiles of 1 << shift pixels.
__device__ __forceinline__ void bbox_tile_rect(uint2 bb, int grid_x, int grid_y, int shift,
                                               int& tx0, int& ty0, int& tx1, int& ty1) {
  tx0 = max(0, min(grid_x - 1, (int)(bb_xmin(bb) >> shift)));
  ty0 = max(0, min(grid_y - 1, (int)(bb_ymin(bb) >> shift)));
  tx1 = max(0, min(grid_x - 1, (int)(bb_xmax(bb) >> shift)));
  ty1 = max(0, min(grid_y - 1, (int)(bb_ymax(bb) >> shift)));
}

__device__ __forceinline__ bool pixel_in_bbox(uint32_t px, uint32_t py, uint2 bb) {
  return px >= bb_xmin(bb) && py >= bb_ymin(bb) && px <= bb_xmax(bb) && py <= bb_ymax(bb);
}

// Octant of a ray direction / of a point relative to the camera origin
// (auxiliary.h:65-73).
__device__ __forceinline__ uint32_t ray_quadrant(float dx, float dy, float dz) {
  return ((uint32_t)(dx < 0.f) << 2) | ((uint32_t)(dy < 0.f) << 1) | (uint32_t)(dz < 0.f);
}

// exp_linear_11 density activation and its derivative (auxiliary.h:278-286).
__device__ __forceinline__ float density_act(float x) {
  return (x > 1.1f) ? x : expf(0.909090909091f * x - 0.904689820196f);
}
__device__ __forceinline__ float density_act_grad(float x) {
  return (x > 1.1f) ? 1.0f : 0.909090909091f * expf(0.909090909091f * x - 0.904689820196f);
}

// Both at once from a single expf: the same exponential the two functions
// above evaluate separately, so the values are identical.
__device__ __forceinline__ void density_act_and_grad(float x, float& act, float& grad) {
  if (x > 1.1f) {
    act = x;
    grad = 1.0f;
  } else {
    const float e = expf(0.909090909091f * x - 0.904689820196f);
    act = e;
    grad = 0.909090909091f * e;
  }
}

// Arithmetic of the compositing loops.  EXACT is the reference's own
// operations (IEEE division, libdevice expf): contributor counts and images
// come out bit-identical.  FAST uses the hardware exponential (ex2.approx of
// x*log2(e), a few ulp) and an approximate division (reciprocal and multiply,
// 2 ulp) for the per-(pixel, voxel) exponentials and the transmittance
// recovery; results then differ from EXACT in the last bits, and a pixel may
// stop one voxel earlier or later where T lands on the early-stop threshold.
template <bool FAST>
__device__ __forceinline__ float exp_f(float x) {
  return FAST ? __expf(x) : expf(x);
}
template <bool FAST>
__device__ __forceinline__ float div_f(float a, float b) {
  return FAST ? __fdividef(a, b) : a / b;
}
template <bool FAST>
__device__ __forceinline__ float density_act_f(float x) {
  return (x > 1.1f) ? x : exp_f<FAST>(0.909090909091f * x - 0.904689820196f);
}
template <bool FAST>
__device__ __forceinline__ void density_act_and_grad_f(float x, float& act, float& grad) {
  if (x > 1.1f) {
    act = x;
    grad = 1.0f;
  } else {
    const float e = exp_f<FAST>(0.909090909091f * x - 0.904689820196f);
    act = e;
    grad = 0.909090909091f * e;
  }
}

__device__ __forceinline__ float contract_depth(float x) {  // auxiliary.h:235-238
  return (x < 1.f) ? x : 2.f - 1.f / x;
}

__device__ __forceinline__ float safe_rnorm3(float x, float y, float z) {
  return rsqrtf(x * x + y * y + z * z + 1e-15f);
}

// Trilinear corner weights, corner index = (ix<<2)|(iy<<1)|iz (auxiliary.h:308-321).
__device__ __forceinline__ void trilinear_weights(float qx, float qy, float qz, float w[8]) {
  const float wx0 = 1.f - qx, wy0 = 1.f - qy, wz0 = 1.f - qz;
  w[0] = wx0 * wy0 * wz0;
  w[1] = wx0 * wy0 * qz;
  w[2] = wx0 * qy * wz0;
  w[3] = wx0 * qy * qz;
  w[4] = qx * wy0 * wz0;
  w[5] = qx * wy0 * qz;
  w[6] = qx * qy * wz0;
  w[7] = qx * qy * qz;
}

// Per-pixel camera ray, identical operation order to forward.cu:103-109 and
// auxiliary.h:76-84.
struct PixelRay {
  float ox, oy, oz;      // origin (camera centre)
  float dx, dy, dz;      // unit direction (world)
  float ix, iy, iz;      // 1 / direction
  float rd_norm_inv;     // 1 / |camera-space direction|
  uint32_t quad;         // octant of the direction
};

__device__ __forceinline__ PixelRay make_pixel_ray(float pixx, float pixy, int W, int H,
                                                   float tanfovx, float tanfovy, float cx, float cy,
                                                   const float* c2w) {
  PixelRay r;
  const float cdx = (pixx + 0.5f - cx) * 2.f * tanfovx / (float)W;
  const float cdy = (pixy + 0.5f - cy) * 2.f * tanfovy / (float)H;
  const float cdz = 1.f;
  // |rd|^2 with the y term fused onto the x product: the reference build
  // evaluates its dot() in this order, and leaving the contraction to the
  // compiler here picks the other operand (measured: images then differ
  // from the reference's in a few ulp at some pixels).
  const float rd_norm = sqrtf(__fmaf_rn(cdy, cdy, __fmul_rn(cdx, cdx)) + cdz * cdz);
  const float rx = c2w[0] * cdx + c2w[1] * cdy + c2w[2] * cdz;
  const float ry = c2w[4] * cdx + c2w[5] * cdy + c2w[6] * cdz;
  const float rz = c2w[8] * cdx + c2w[9] * cdy + c2w[10] * cdz;
  r.rd_norm_inv = 1.f / rd_norm;
  r.ox = c2w[3];
  r.oy = c2w[7];
  r.oz = c2w[11];
  r.dx = rx * r.rd_norm_inv;
  r.dy = ry * r.rd_norm_inv;
  r.dz = rz * r.rd_norm_inv;
  r.ix = 1.f / r.dx;
  r.iy = 1.f / r.dy;
  r.iz = 1.f / r.dz;
  r.quad = ray_quadrant(r.dx, r.dy, r.dz);
  return r;
}

// Slab test of a ray against an axis-aligned voxel (auxiliary.h:240-253).
__device__ __forceinline__ float2 ray_box(float cx, float cy, float cz, float len, const PixelRay& r) {
  const float rad = 0.5f * len;
  const float dx = cx - r.ox, dy = cy - r.oy, dz = cz - r.oz;
  const float ax = (dx - rad) * r.ix, ay = (dy - rad) * r.iy, az = (dz - rad) * r.iz;
  const float bx = (dx + rad) * r.ix, by = (dy + rad) * r.iy, bz = (dz + rad) * r.iz;
  const float nx = fminf(ax, bx), ny = fminf(ay, by), nz = fminf(az, bz);
  const float fx = fmaxf(ax, bx), fy = fmaxf(ay, by), fz = fmaxf(az, bz);
  return make_float2(fmaxf(fmaxf(nx, ny), nz), fminf(fminf(fx, fy), fz));
}


}  // namespace svr
