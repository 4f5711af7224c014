// Backward compositing kernels and their template dispatch: the plain
// one-view grid (16x16 tiles) and the multi-view persistent form (tile size
// and staging depth chosen per plan).
#include <mutex>

#include "svr_kernels.h"
#include "svr_render_bwd.cuh"
#include "svr_render_pair.cuh"

namespace svr {

struct BwdArgs {
  ViewParams vp;
  const uint2* ranges;
  const uint32_t* tile_last;
  const uint32_t* vals;
  VoxelArrays va;
  BwdTileIn in;
  BwdTileOut out;
  const uint32_t* order;  // CTA i renders tile order[i] (identity when null)
};

template <class CFG>
struct BwdSmem {
  StageSmem<CFG::SB> s;
  float grad[GradAcc<CFG>::kFloats];
  uint32_t hit[GradAcc<CFG>::kWords];
  float c2w[12];
  uint32_t item;
};

// CTA b back-propagates quadrant b % 4 of the 16x16 list order[b / 4].
template <int NS, bool DEPTH, bool DIST, bool NORMAL>
__global__ void __launch_bounds__(PlainTile::NT, (bwd_min_blocks_for<PlainTile, DIST>()))
render_bwd_kernel(const __grid_constant__ BwdArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BwdSmem<PlainTile>& sm = *reinterpret_cast<BwdSmem<PlainTile>*>(smem_raw);
  if (threadIdx.x < 12) sm.c2w[threadIdx.x] = a.vp.c2w[threadIdx.x];
  __syncthreads();
  const int b = blockIdx.x / kPlainSub, sub = blockIdx.x % kPlainSub;
  const int tile = a.order ? (int)a.order[b] : b;
  const int tile_x = (tile % a.vp.grid_x) * 2 + (sub & 1), tile_y = (tile / a.vp.grid_x) * 2 + (sub >> 1);
  render_tile_bwd<PlainTile, NS, DEPTH, DIST, NORMAL>(a.vp, sm.c2w, tile_x, tile_y, a.ranges[tile], a.tile_last[tile],
                                                      a.vals, a.va, a.in, a.out, sm.s, sm.grad, sm.hit);
}

// Multi-view form: a persistent grid over all views' tiles, in the order of
// `order` (see the forward's FwdBatchArgs).
struct BwdBatchArgs {
  ViewTable views;
  int n_items;
  const uint2* ranges;
  const uint32_t* tile_last;
  const uint32_t* vals;
  VoxelArrays va;
  int P;
  size_t rgb_view_stride;   // elements between views in va.rgbs ([V,P,3])
  size_t drgb_view_stride;  // elements between views in out.dL_drgbs ([V,P,4])
  BwdTileIn in;    // base pointers, offset per view
  BwdTileOut out;  // dL_drgbs offset per view by drgb_view_stride
  const uint32_t* order;  // [n_items] work order, or nullptr
  uint32_t* counter;      // work counter, zero at launch
};

template <class CFG, int NS, bool FAST>
__global__ void __launch_bounds__(CFG::NT, bwd_min_blocks<CFG>())
render_bwd_batch_kernel(const __grid_constant__ BwdBatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BwdSmem<CFG>& sm = *reinterpret_cast<BwdSmem<CFG>*>(smem_raw);
  for (;;) {
    if (threadIdx.x == 0) sm.item = atomicAdd(a.counter, 1u);
    __syncthreads();
    const uint32_t k = sm.item;
    if (k >= (uint32_t)a.n_items) break;
    const int item = a.order ? (int)a.order[k] : (int)k;
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
    BwdTileOut o = a.out;
    o.dL_drgbs = a.out.dL_drgbs + (size_t)view * a.drgb_view_stride;
    render_tile_bwd<CFG, NS, false, false, false, FAST, true>(vp, sm.c2w, tile_x, tile_y, a.ranges[item],
                                                              a.tile_last[item], a.vals, va, in, o, sm.s, sm.grad, sm.hit);
    __syncthreads();  // shared state (item, camera, staging) is free for the next tile
  }
}

// The same persistent form with two pixels per thread (svr_render_pair.cuh).
template <class CFG, int NS, bool FAST, bool GRID>
__global__ void __launch_bounds__(CFG::NT, pair_min_blocks<CFG>())
render_bwd_batch_pair_kernel(const __grid_constant__ BwdBatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BwdSmem<CFG>& sm = *reinterpret_cast<BwdSmem<CFG>*>(smem_raw);
  for (;;) {
    if (threadIdx.x == 0) sm.item = atomicAdd(a.counter, 1u);
    __syncthreads();
    const uint32_t k = sm.item;
    if (k >= (uint32_t)a.n_items) break;
    const int item = a.order ? (int)a.order[k] : (int)k;
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
    BwdTileOut o = a.out;
    o.dL_drgbs = a.out.dL_drgbs + (size_t)view * a.drgb_view_stride;
    render_tile_bwd_pair<CFG, NS, FAST, GRID>(vp, sm.c2w, tile_x, tile_y, a.ranges[item], a.tile_last[item], a.vals, va,
                                        in, o, sm.s, sm.grad, sm.hit);
    __syncthreads();
  }
}

static_assert(sizeof(BwdSmem<PlainTile>) <= 48 * 1024, "plain backward staging must fit the default limit");

#define SVR_BWD_CASE(KERNEL, NS_, D_, T_, N_)                                                     \
  if (ns == NS_ && depth == D_ && dist == T_ && normal == N_) {                                   \
    KERNEL<NS_, D_, T_, N_><<<grid, PlainTile::NT, sizeof(BwdSmem<PlainTile>), stream>>>(args);   \
    return;                                                                                       \
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
                       bool dist, bool normal, const uint32_t* order, cudaStream_t stream) {
  BwdArgs args{vp, ranges, tile_last, vals, va, in, out, order};
  const dim3 grid(vp.grid_x * vp.grid_y * kPlainSub);
  SVR_BWD_SWITCH(render_bwd_kernel)
}

template <class CFG>
static void set_bwd_pair_attrs() {
  const int smem = (int)sizeof(BwdSmem<CFG>);
  auto set = [smem](const void* k) { cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); };
  set((const void*)render_bwd_batch_pair_kernel<CFG, 1, false, false>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 2, false, false>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 3, false, false>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 1, true, false>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 2, true, false>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 3, true, false>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 1, false, true>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 2, false, true>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 3, false, true>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 1, true, true>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 2, true, true>);
  set((const void*)render_bwd_batch_pair_kernel<CFG, 3, true, true>);
}

template <class CFG, int NS>
static void set_bwd_batch_attr() {
  cudaFuncSetAttribute(render_bwd_batch_kernel<CFG, NS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BwdSmem<CFG>));
  cudaFuncSetAttribute(render_bwd_batch_kernel<CFG, NS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BwdSmem<CFG>));
}

template <class CFG>
static void set_bwd_batch_attrs() {
  set_bwd_batch_attr<CFG, 1>();
  set_bwd_batch_attr<CFG, 2>();
  set_bwd_batch_attr<CFG, 3>();
}

void ensure_bwd_batch_attributes() {
  static std::once_flag flags[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  std::call_once(flags[dev], [] {
    set_bwd_batch_attrs<TileCfg<16, 128>>();
    set_bwd_batch_attrs<TileCfg<16, 256>>();
    set_bwd_batch_attrs<TileCfg<16, 512>>();
    set_bwd_batch_attrs<TileCfg<8, 32>>();
    set_bwd_batch_attrs<TileCfg<8, 64>>();
    set_bwd_batch_attrs<TileCfg<8, 128>>();
    set_bwd_batch_attrs<TileCfg<32, 256>>();
    set_bwd_pair_attrs<PairCfg<8, 32>>();
    set_bwd_pair_attrs<PairCfg<8, 64>>();
    set_bwd_pair_attrs<PairCfg<16, 128>>();
    set_bwd_pair_attrs<PairCfg<16, 256>>();
  });
}

template <class CFG, bool FAST>
static void launch_bwd_batch_arith(const BwdBatchArgs& args, int ns, int ctas_per_sm, cudaStream_t stream) {
  const size_t smem = sizeof(BwdSmem<CFG>);
  auto go = [&](auto kfn) {
    const int grid = persistent_grid((const void*)kfn, CFG::NT, smem, args.n_items, ctas_per_sm);
    kfn<<<grid, CFG::NT, smem, stream>>>(args);
  };
  if (ns == 1) go(render_bwd_batch_kernel<CFG, 1, FAST>);
  else if (ns == 2) go(render_bwd_batch_kernel<CFG, 2, FAST>);
  else go(render_bwd_batch_kernel<CFG, 3, FAST>);
}

template <class CFG, bool FAST>
static void launch_bwd_pair_arith(const BwdBatchArgs& args, int ns, int ctas_per_sm, cudaStream_t stream) {
  const size_t smem = sizeof(BwdSmem<CFG>);
  auto go = [&](auto kfn) {
    const int grid = persistent_grid((const void*)kfn, CFG::NT, smem, args.n_items, ctas_per_sm);
    kfn<<<grid, CFG::NT, smem, stream>>>(args);
  };
  const bool grid = args.va.key != nullptr;
  if (ns == 1) grid ? go(render_bwd_batch_pair_kernel<CFG, 1, FAST, true>) : go(render_bwd_batch_pair_kernel<CFG, 1, FAST, false>);
  else if (ns == 2) grid ? go(render_bwd_batch_pair_kernel<CFG, 2, FAST, true>) : go(render_bwd_batch_pair_kernel<CFG, 2, FAST, false>);
  else grid ? go(render_bwd_batch_pair_kernel<CFG, 3, FAST, true>) : go(render_bwd_batch_pair_kernel<CFG, 3, FAST, false>);
}

template <class CFG>
static void launch_bwd_pair_cfg(const BwdBatchArgs& args, int ns, bool fast, int ctas_per_sm, cudaStream_t stream) {
  if (fast) launch_bwd_pair_arith<CFG, true>(args, ns, ctas_per_sm, stream);
  else launch_bwd_pair_arith<CFG, false>(args, ns, ctas_per_sm, stream);
}

template <class CFG>
static void launch_bwd_batch_cfg(const BwdBatchArgs& args, int ns, bool fast, int ctas_per_sm, cudaStream_t stream) {
  if (fast) launch_bwd_batch_arith<CFG, true>(args, ns, ctas_per_sm, stream);
  else launch_bwd_batch_arith<CFG, false>(args, ns, ctas_per_sm, stream);
}

void launch_render_bwd_batch(const ViewTable& views, int n_items, const uint2* ranges,
                             const uint32_t* tile_last, const uint32_t* vals, const VoxelArrays& va, int P,
                             size_t rgb_view_stride, size_t drgb_view_stride, const BwdTileIn& in,
                             const BwdTileOut& out, int ns, int tile, int stage, bool fast, int pair,
                             const uint32_t* order, uint32_t* counter, int ctas_per_sm, cudaStream_t stream) {
  if (n_items <= 0) return;
  ensure_bwd_batch_attributes();
  cudaMemsetAsync(counter, 0, sizeof(uint32_t), stream);
  const BwdBatchArgs args{views, n_items, ranges, tile_last, vals, va, P, rgb_view_stride, drgb_view_stride, in, out,
                          order, counter};
  if (pair && batch_pair_supported(tile, stage)) {
    if (tile == 8 && stage == 32) launch_bwd_pair_cfg<PairCfg<8, 32>>(args, ns, fast, ctas_per_sm, stream);
    else if (tile == 8) launch_bwd_pair_cfg<PairCfg<8, 64>>(args, ns, fast, ctas_per_sm, stream);
    else if (stage == 128) launch_bwd_pair_cfg<PairCfg<16, 128>>(args, ns, fast, ctas_per_sm, stream);
    else launch_bwd_pair_cfg<PairCfg<16, 256>>(args, ns, fast, ctas_per_sm, stream);
    return;
  }
  if (tile == 8 && stage == 32) launch_bwd_batch_cfg<TileCfg<8, 32>>(args, ns, fast, ctas_per_sm, stream);
  else if (tile == 8 && stage == 128) launch_bwd_batch_cfg<TileCfg<8, 128>>(args, ns, fast, ctas_per_sm, stream);
  else if (tile == 8) launch_bwd_batch_cfg<TileCfg<8, 64>>(args, ns, fast, ctas_per_sm, stream);
  else if (tile == 32) launch_bwd_batch_cfg<TileCfg<32, 256>>(args, ns, fast, ctas_per_sm, stream);
  else if (stage == 128) launch_bwd_batch_cfg<TileCfg<16, 128>>(args, ns, fast, ctas_per_sm, stream);
  else if (stage == 512) launch_bwd_batch_cfg<TileCfg<16, 512>>(args, ns, fast, ctas_per_sm, stream);
  else launch_bwd_batch_cfg<TileCfg<16, 256>>(args, ns, fast, ctas_per_sm, stream);
}

}  // namespace svr
