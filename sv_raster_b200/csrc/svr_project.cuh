// Projection of one voxel into one view: near-sphere cull, 8 corners to a
// packed pixel bbox, camera-quadrant bitset and duplicate count.
//
// Same arithmetic as preprocessCUDA (backends/cuda/src/preprocess.cu:54-131).
// The reference traps when the tile count is not positive
// (preprocess.cu:119-124); that cannot happen here because the bbox test
// guarantees min <= max, so the clamped tile rectangle is never empty.
#pragma once

#include "svr_common.cuh"
#include "svr_views.cuh"

namespace svr {

struct Projection {
  uint32_t n;      // tiles touched x quadrants touched (0 = culled)
  uint2 bbox;      // packed pixel bbox
  uint32_t quads;  // camera-quadrant bitset (0 when culled)
  float bx0, by0, bx1, by1;  // the bbox before rounding (pixel coordinates, clamped to the image)
  bool front;                // all 8 corners in front of the near plane
};

__device__ __forceinline__ Projection project_voxel(const ViewParams& vp, const float* w2c, const float* c2w,
                                                    float vcx, float vcy, float vcz, float len) {
  Projection pr{0u, make_uint2(0u, 0u), 0u, 0.f, 0.f, 0.f, 0.f, false};
  const float vr = 0.5f * len;
  const float rox = c2w[3], roy = c2w[7], roz = c2w[11];
  const float near = vp.near_plane;
  const float rx = vcx - rox, ry = vcy - roy, rz = vcz - roz;
  if (rx * rx + ry * ry + rz * rz < near * near) return pr;
  float umin = 1e9f, vmin = 1e9f, umax = -1e9f, vmax = -1e9f;
  uint32_t qbits = 0;
  int n_front = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float sx = (float)(((i & 4) >> 2) * 2 - 1);
    const float sy = (float)(((i & 2) >> 1) * 2 - 1);
    const float sz = (float)(((i & 1)) * 2 - 1);
    const float wx = vcx + vr * sx, wy = vcy + vr * sy, wz = vcz + vr * sz;
    const float camx = w2c[0] * wx + w2c[1] * wy + w2c[2] * wz + w2c[3];
    const float camy = w2c[4] * wx + w2c[5] * wy + w2c[6] * wz + w2c[7];
    const float camz = w2c[8] * wx + w2c[9] * wy + w2c[10] * wz + w2c[11];
    if (camz < near) continue;
    const float inv_z = 1.0f / camz;
    const float u = camx * inv_z, v = camy * inv_z;
    const uint32_t q = ((uint32_t)(wx < rox) << 2) | ((uint32_t)(wy < roy) << 1) | (uint32_t)(wz < roz);
    umin = fminf(umin, u); vmin = fminf(vmin, v);
    umax = fmaxf(umax, u); vmax = fmaxf(vmax, v);
    qbits |= (1u << q);
    ++n_front;
  }
  const float cxh = vp.cx - 0.5f, cyh = vp.cy - 0.5f;
  const float bx0 = fmaxf(vp.focal_x * umin + cxh, 0.0f);
  const float by0 = fmaxf(vp.focal_y * vmin + cyh, 0.0f);
  const float bx1 = fminf(vp.focal_x * umax + cxh, (float)vp.W);
  const float by1 = fminf(vp.focal_y * vmax + cyh, (float)vp.H);
  if (bx0 > bx1 || by0 > by1) return pr;
  pr.bbox.x = (((uint32_t)lrintf(bx0)) << 16) | ((uint32_t)lrintf(by0));
  pr.bbox.y = (((uint32_t)lrintf(bx1)) << 16) | ((uint32_t)lrintf(by1));
  int tx0, ty0, tx1, ty1;
  bbox_tile_rect(pr.bbox, vp.grid_x, vp.grid_y, vp.tile_shift, tx0, ty0, tx1, ty1);
  pr.n = (uint32_t)((1 + ty1 - ty0) * (1 + tx1 - tx0)) * (uint32_t)__popc(qbits);
  pr.quads = qbits;
  pr.bx0 = bx0; pr.by0 = by0; pr.bx1 = bx1; pr.by1 = by1;
  pr.front = n_front == 8;
  return pr;
}

// The pixels of the rounded bbox whose centre ray can meet the cube.  The ray
// of pixel (px, py) has the projected coordinates (px, py) themselves (the
// ray direction of make_pixel_ray, (p + 0.5 - c) / focal, maps to
// focal * u + c - 0.5 = p), and with all 8 corners in front of the near plane
// the cube's image is the convex hull of its projected corners, inside the
// unrounded bbox.  The rounded bbox (lrintf of each side) can hold one more
// pixel per side whose ray misses; for a sub-pixel voxel the unrounded bbox
// often holds no pixel centre at all.  A margin of kTightMargin pixels keeps
// rays that rounding could put on the cube's silhouette (such a ray crosses
// a vanishing chord and contributes nothing either way).  Voxels with a corner
// behind the near plane keep the rounded bbox.  Returns false when no pixel
// centre remains (the voxel is culled for this view).
constexpr float kTightMargin = 0.05f;

__device__ __forceinline__ bool tighten_bbox(const ViewParams& vp, Projection& pr) {
  if (pr.n == 0 || !pr.front) return pr.n != 0;
  const int x0 = max((int)bb_xmin(pr.bbox), (int)ceilf(pr.bx0 - kTightMargin));
  const int y0 = max((int)bb_ymin(pr.bbox), (int)ceilf(pr.by0 - kTightMargin));
  const int x1 = min((int)bb_xmax(pr.bbox), (int)floorf(pr.bx1 + kTightMargin));
  const int y1 = min((int)bb_ymax(pr.bbox), (int)floorf(pr.by1 + kTightMargin));
  if (x0 > x1 || y0 > y1) {
    pr.n = 0;
    pr.quads = 0;
    pr.bbox = make_uint2(0u, 0u);
    return false;
  }
  pr.bbox.x = ((uint32_t)x0 << 16) | (uint32_t)y0;
  pr.bbox.y = ((uint32_t)x1 << 16) | (uint32_t)y1;
  int tx0, ty0, tx1, ty1;
  bbox_tile_rect(pr.bbox, vp.grid_x, vp.grid_y, vp.tile_shift, tx0, ty0, tx1, ty1);
  pr.n = (uint32_t)((1 + ty1 - ty0) * (1 + tx1 - tx0)) * (uint32_t)__popc(pr.quads);
  return true;
}

}  // namespace svr
