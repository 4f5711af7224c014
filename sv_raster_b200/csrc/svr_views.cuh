// Per-view camera description passed to every kernel by value.
#pragma once

#include <cstdint>

namespace svr {

constexpr int kMaxViews = 64;

struct ViewParams {
  int W, H;              // image size in pixels
  int grid_x, grid_y;    // tile grid (ceil(W/ts), ceil(H/ts)), ts = 1 << tile_shift
  int tile_shift;        // log2 of the tile size (4 on the plain path)
  float tanfovx, tanfovy;
  float cx, cy;          // principal point in pixels
  float focal_x, focal_y;  // 0.5*W/tanfovx, computed in float on the host (preprocess.cu:173-174)
  float near_plane;
  float bg;              // background intensity
  const float* w2c;      // device, row-major 4x4 (first 12 read)
  const float* c2w;      // device, row-major 4x4 (first 12 read)
  uint32_t tile_base;    // first global tile id of this view (batched path)
  uint32_t pix_base;     // first global pixel of this view (batched path)
  uint32_t sort_tile_off;  // tile id offset of this view inside its sort group
  int sort_group;          // sort group of this view
};

struct ViewTable {
  int n;
  ViewParams v[kMaxViews];
};

// View owning global tile `item` (views are laid out by ascending tile_base).
__device__ __forceinline__ int view_of_tile(const ViewTable& t, int item) {
  int lo = 0, hi = t.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((int)t.v[mid].tile_base <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

}  // namespace svr
