// Forward compositing kernels (plain one-view grid and the multi-view form,
// one CTA per (view, tile) of every view in a single launch) and their
// template dispatch.
#include "svr_kernels.h"
#include "svr_render_fwd.cuh"

namespace svr {

struct FwdArgs {
  ViewParams vp;
  const uint2* ranges;
  const uint32_t* vals;
  VoxelArrays va;
  FwdTileOut out;
};

template <int NS, bool DEPTH, bool DIST, bool NORMAL, bool MAXW>
__global__ void __launch_bounds__(kBatch, kFwdMinBlocks)
render_fwd_kernel(const __grid_constant__ FwdArgs a) {
  __shared__ StageSmem s;
  __shared__ float s_c2w[12];
  __shared__ uint32_t s_red[kBatch / 32];
  if (threadIdx.x < 12) s_c2w[threadIdx.x] = a.vp.c2w[threadIdx.x];
  __syncthreads();
  const int tile_x = blockIdx.x, tile_y = blockIdx.y;
  const uint2 range = a.ranges[tile_y * a.vp.grid_x + tile_x];
  render_tile_fwd<NS, DEPTH, DIST, NORMAL, MAXW>(a.vp, s_c2w, tile_x, tile_y, range, a.vals, a.va, a.out, s, s_red);
}

// Multi-view form: one CTA per (view, tile) work item, items laid out view by
// view.  Per-view arrays are addressed through the view's tile/pixel bases.
struct FwdBatchArgs {
  ViewTable views;
  int n_items;                 // total tiles over all views
  const uint2* ranges;         // [sum T]
  const uint32_t* vals;        // sorted values, per-view segments (absolute offsets in ranges)
  VoxelArrays va;              // bboxes / rgbs are [V,P] (offset per view below)
  int P;
  size_t rgb_view_stride;      // elements between views in rgbs (0 = shared)
  FwdTileOut out;              // base pointers; offset per view
};

template <int NS, bool DEPTH, bool DIST, bool NORMAL, bool MAXW>
__global__ void __launch_bounds__(kBatch, kFwdMinBlocks)
render_fwd_batch_kernel(const __grid_constant__ FwdBatchArgs a) {
  __shared__ StageSmem s;
  __shared__ float s_c2w[12];
  __shared__ uint32_t s_red[kBatch / 32];
  const int item = blockIdx.x;
  if (item >= a.n_items) return;
  const int view = view_of_tile(a.views, item);
  const ViewParams& vp = a.views.v[view];
  if (threadIdx.x < 12) s_c2w[threadIdx.x] = vp.c2w[threadIdx.x];
  __syncthreads();
  const int local = item - (int)vp.tile_base;
  const int tile_x = local % vp.grid_x, tile_y = local / vp.grid_x;
  const uint2 range = a.ranges[item];
  VoxelArrays va = a.va;
  va.bboxes = a.va.bboxes + (size_t)view * a.P;
  va.rgbs = a.va.rgbs + (size_t)view * a.rgb_view_stride;
  FwdTileOut o = a.out;
  o.tile_last = a.out.tile_last + vp.tile_base;
  o.n_contrib = a.out.n_contrib + vp.pix_base;
  o.color = a.out.color + 3 * (size_t)vp.pix_base;
  o.T = a.out.T + vp.pix_base;
  if (DEPTH || DIST) o.depth = a.out.depth + 3 * (size_t)vp.pix_base;
  if (NORMAL) o.normal = a.out.normal + 3 * (size_t)vp.pix_base;
  if (MAXW) o.max_w = a.out.max_w + (size_t)view * a.P;
  render_tile_fwd<NS, DEPTH, DIST, NORMAL, MAXW>(vp, s_c2w, tile_x, tile_y, range, a.vals, va, o, s, s_red);
}

#define SVR_FWD_DISPATCH(KERNEL, GRID, STREAM, ...)                                                   \
  do {                                                                                                \
    const int _ns = ns;                                                                               \
    const bool _d = depth, _t = dist, _n = normal, _m = maxw;                                         \
    auto _launch = [&](auto kfn) { kfn<<<GRID, kBatch, 0, STREAM>>>(__VA_ARGS__); };                  \
    (void)_launch;                                                                                    \
    SVR_FWD_SWITCH(KERNEL, _ns, _d, _t, _n, _m);                                                      \
  } while (0)

#define SVR_FWD_CASE(KERNEL, NS_, D_, T_, N_, M_) \
  if (_ns == NS_ && _d == D_ && _t == T_ && _n == N_ && _m == M_) { _launch(KERNEL<NS_, D_, T_, N_, M_>); break; }

#define SVR_FWD_CASES_NS(KERNEL, NS_)                                                              \
  SVR_FWD_CASE(KERNEL, NS_, false, false, false, false) SVR_FWD_CASE(KERNEL, NS_, false, false, false, true) \
  SVR_FWD_CASE(KERNEL, NS_, false, false, true, false) SVR_FWD_CASE(KERNEL, NS_, false, false, true, true)   \
  SVR_FWD_CASE(KERNEL, NS_, false, true, false, false) SVR_FWD_CASE(KERNEL, NS_, false, true, false, true)   \
  SVR_FWD_CASE(KERNEL, NS_, false, true, true, false) SVR_FWD_CASE(KERNEL, NS_, false, true, true, true)     \
  SVR_FWD_CASE(KERNEL, NS_, true, false, false, false) SVR_FWD_CASE(KERNEL, NS_, true, false, false, true)   \
  SVR_FWD_CASE(KERNEL, NS_, true, false, true, false) SVR_FWD_CASE(KERNEL, NS_, true, false, true, true)     \
  SVR_FWD_CASE(KERNEL, NS_, true, true, false, false) SVR_FWD_CASE(KERNEL, NS_, true, true, false, true)     \
  SVR_FWD_CASE(KERNEL, NS_, true, true, true, false) SVR_FWD_CASE(KERNEL, NS_, true, true, true, true)

#define SVR_FWD_SWITCH(KERNEL, ...)                                                 \
  for (;;) {                                                                        \
    SVR_FWD_CASES_NS(KERNEL, 1) SVR_FWD_CASES_NS(KERNEL, 2) SVR_FWD_CASES_NS(KERNEL, 3) \
    break;                                                                          \
  }

void launch_render_fwd(const ViewParams& vp, const uint2* ranges, const uint32_t* vals, const VoxelArrays& va,
                       const FwdTileOut& out, int ns, bool depth, bool dist, bool normal, bool maxw,
                       cudaStream_t stream) {
  FwdArgs args{vp, ranges, vals, va, out};
  dim3 grid(vp.grid_x, vp.grid_y);
  SVR_FWD_DISPATCH(render_fwd_kernel, grid, stream, args);
}

void launch_render_fwd_batch(const ViewTable& views, int n_items, const uint2* ranges,
                             const uint32_t* vals, const VoxelArrays& va, int P, size_t rgb_view_stride,
                             const FwdTileOut& out, int ns, bool depth, bool dist, bool normal, bool maxw,
                             cudaStream_t stream) {
  if (n_items <= 0) return;
  FwdBatchArgs args{views, n_items, ranges, vals, va, P, rgb_view_stride, out};
  dim3 grid(n_items);
  SVR_FWD_DISPATCH(render_fwd_batch_kernel, grid, stream, args);
}

}  // namespace svr
