// Backward compositing kernels (plain one-view grid and the multi-view form)
// and their template dispatch.
#include "svr_kernels.h"
#include "svr_render_bwd.cuh"

namespace svr {

struct BwdArgs {
  ViewParams vp;
  const uint2* ranges;
  const uint32_t* tile_last;
  const uint32_t* vals;
  VoxelArrays va;
  BwdTileIn in;
  BwdTileOut out;
};

struct BwdSmem {
  StageSmem s;
  float grad[kBatch * kGradStride];
  float c2w[12];
};

template <int NS, bool DEPTH, bool DIST, bool NORMAL>
__global__ void __launch_bounds__(kBatch, kBwdMinBlocks)
render_bwd_kernel(const __grid_constant__ BwdArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BwdSmem& sm = *reinterpret_cast<BwdSmem*>(smem_raw);
  if (threadIdx.x < 12) sm.c2w[threadIdx.x] = a.vp.c2w[threadIdx.x];
  __syncthreads();
  const int tile_x = blockIdx.x, tile_y = blockIdx.y;
  const int tile = tile_y * a.vp.grid_x + tile_x;
  render_tile_bwd<NS, DEPTH, DIST, NORMAL>(a.vp, sm.c2w, tile_x, tile_y, a.ranges[tile], a.tile_last[tile], a.vals,
                                           a.va, a.in, a.out, sm.s, sm.grad);
}

struct BwdBatchArgs {
  ViewTable views;
  int n_items;
  const uint2* ranges;
  const uint32_t* tile_last;
  const uint32_t* vals;
  VoxelArrays va;
  int P;
  size_t rgb_view_stride;
  BwdTileIn in;    // base pointers, offset per view
  BwdTileOut out;  // dL_drgbs offset per view by rgb_view_stride
};

template <int NS, bool DEPTH, bool DIST, bool NORMAL>
__global__ void __launch_bounds__(kBatch, kBwdMinBlocks)
render_bwd_batch_kernel(const __grid_constant__ BwdBatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BwdSmem& sm = *reinterpret_cast<BwdSmem*>(smem_raw);
  const int item = blockIdx.x;
  if (item >= a.n_items) return;
  const int view = view_of_tile(a.views, item);
  const ViewParams& vp = a.views.v[view];
  if (threadIdx.x < 12) sm.c2w[threadIdx.x] = vp.c2w[threadIdx.x];
  __syncthreads();
  const int local = item - (int)vp.tile_base;
  const int tile_x = local % vp.grid_x, tile_y = local / vp.grid_x;
  VoxelArrays va = a.va;
  va.bboxes = a.va.bboxes + (size_t)view * a.P;
  va.rgbs = a.va.rgbs + (size_t)view * a.rgb_view_stride;
  BwdTileIn in = a.in;
  const size_t pb = vp.pix_base;
  in.T = a.in.T + pb;
  in.n_contrib = a.in.n_contrib + pb;
  in.dL_dcolor = a.in.dL_dcolor + 3 * pb;
  in.dL_dT = a.in.dL_dT + pb;
  if (DEPTH) in.dL_ddepth = a.in.dL_ddepth + 3 * pb;
  if (NORMAL) in.dL_dnormal = a.in.dL_dnormal + 3 * pb;
  if (a.in.gt_color) in.gt_color = a.in.gt_color + 3 * pb;
  if (a.in.out_depth) in.out_depth = a.in.out_depth + 3 * pb;
  BwdTileOut o = a.out;
  o.dL_drgbs = a.out.dL_drgbs + (size_t)view * a.rgb_view_stride;
  render_tile_bwd<NS, DEPTH, DIST, NORMAL>(vp, sm.c2w, tile_x, tile_y, a.ranges[item], a.tile_last[item], a.vals, va,
                                           in, o, sm.s, sm.grad);
}

static_assert(sizeof(BwdSmem) <= 48 * 1024, "backward staging must fit the default shared-memory limit");

#define SVR_BWD_CASE(KERNEL, NS_, D_, T_, N_)                                    \
  if (ns == NS_ && depth == D_ && dist == T_ && normal == N_) {                  \
    KERNEL<NS_, D_, T_, N_><<<grid, kBatch, sizeof(BwdSmem), stream>>>(ARGS);    \
    return;                                                                      \
  }
#define SVR_BWD_CASES_NS(KERNEL, NS_)                                                            \
  SVR_BWD_CASE(KERNEL, NS_, false, false, false) SVR_BWD_CASE(KERNEL, NS_, false, false, true) \
  SVR_BWD_CASE(KERNEL, NS_, false, true, false) SVR_BWD_CASE(KERNEL, NS_, false, true, true)   \
  SVR_BWD_CASE(KERNEL, NS_, true, false, false) SVR_BWD_CASE(KERNEL, NS_, true, false, true)   \
  SVR_BWD_CASE(KERNEL, NS_, true, true, false) SVR_BWD_CASE(KERNEL, NS_, true, true, true)
#define SVR_BWD_SWITCH(KERNEL) \
  SVR_BWD_CASES_NS(KERNEL, 1) SVR_BWD_CASES_NS(KERNEL, 2) SVR_BWD_CASES_NS(KERNEL, 3)

void launch_render_bwd(const ViewParams& vp, const uint2* ranges, const uint32_t* tile_last, const uint32_t* vals,
                       const VoxelArrays& va, const BwdTileIn& in, const BwdTileOut& out, int ns, bool depth,
                       bool dist, bool normal, cudaStream_t stream) {
  BwdArgs args{vp, ranges, tile_last, vals, va, in, out};
  dim3 grid(vp.grid_x, vp.grid_y);
#define ARGS args
  SVR_BWD_SWITCH(render_bwd_kernel)
#undef ARGS
}

void launch_render_bwd_batch(const ViewTable& views, int n_items, const uint2* ranges,
                             const uint32_t* tile_last, const uint32_t* vals, const VoxelArrays& va, int P,
                             size_t rgb_view_stride, const BwdTileIn& in, const BwdTileOut& out, int ns, bool depth,
                             bool dist, bool normal, cudaStream_t stream) {
  if (n_items <= 0) return;
  BwdBatchArgs args{views, n_items, ranges, tile_last, vals, va, P, rgb_view_stride, in, out};
  dim3 grid(n_items);
#define ARGS args
  SVR_BWD_SWITCH(render_bwd_batch_kernel)
#undef ARGS
}

}  // namespace svr
