// Forward compositing kernels and their template dispatch: the plain
// one-view grid (the reference's 16x16 tile lists, four 8x8 CTAs each) and the
// multi-view form (one persistent launch over every (view, tile) of all
// views, tile size and staging depth chosen per plan).
#include <mutex>

#include "svr_kernels.h"
#include "svr_render_fwd.cuh"
#include "svr_render_pair.cuh"

namespace svr {

int persistent_grid(const void* kernel, int threads, size_t dyn_smem, int n_items, int ctas_per_sm) {
  int dev = 0, sms = 1, per_sm = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, dyn_smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  if (ctas_per_sm > 0) per_sm = std::min(per_sm, ctas_per_sm);
  const long long g = (long long)sms * per_sm;
  return (int)std::max(1LL, std::min<long long>(g, (long long)n_items));
}

struct FwdArgs {
  ViewParams vp;
  const uint2* ranges;
  const uint32_t* vals;
  VoxelArrays va;
  FwdTileOut out;
  const uint32_t* order;  // CTA i renders tile order[i] (identity when null)
};

// CTA b composites quadrant b % 4 of the 16x16 list order[b / 4] (the
// caller zeroes tile_last; the four quadrants combine it with atomicMax).
template <int NS, bool DEPTH, bool DIST, bool NORMAL, bool MAXW>
__global__ void __launch_bounds__(PlainTile::NT, fwd_min_blocks<PlainTile>())
render_fwd_kernel(const __grid_constant__ FwdArgs a) {
  __shared__ StageSmem<PlainTile::SB> s;
  __shared__ float s_c2w[12];
  __shared__ uint32_t s_red[PlainTile::NW];
  if (threadIdx.x < 12) s_c2w[threadIdx.x] = a.vp.c2w[threadIdx.x];
  __syncthreads();
  const int b = blockIdx.x / kPlainSub, sub = blockIdx.x % kPlainSub;
  const int tile = a.order ? (int)a.order[b] : b;
  const int tile_x = (tile % a.vp.grid_x) * 2 + (sub & 1), tile_y = (tile / a.vp.grid_x) * 2 + (sub >> 1);
  const uint2 range = a.ranges[tile];
  render_tile_fwd<PlainTile, NS, DEPTH, DIST, NORMAL, MAXW, true>(a.vp, s_c2w, tile_x, tile_y, range, a.vals, a.va,
                                                                  a.out, a.out.tile_last + tile, s, s_red);
}

// Multi-view form: a persistent grid over the (view, tile) work items of all
// views, items laid out view by view.  CTAs take items from a device counter
// in the order of `order` (largest tiles first when the caller ranks them by
// cost; identity when null), so the heavy-tailed tile costs do not leave a
// tail of late large tiles.  Per-view arrays are addressed through the view's
// tile/pixel bases.
struct FwdBatchArgs {
  ViewTable views;
  int n_items;                 // total tiles over all views
  const uint2* ranges;         // [sum T]
  const uint32_t* vals;        // sorted values, per-view segments (absolute offsets in ranges)
  VoxelArrays va;              // bboxes / rgbs are [V,P] (offset per view below)
  int P;
  size_t rgb_view_stride;      // elements between views in rgbs (0 = shared)
  FwdTileOut out;              // base pointers; offset per view
  const uint32_t* order;       // [n_items] work order, or nullptr
  uint32_t* counter;           // work counter, zero at launch
};

template <class CFG>
struct FwdBatchSmem {
  StageSmem<CFG::SB> s;
  float c2w[12];
  uint32_t red[CFG::NW];
  uint32_t item;
};

template <class CFG, int NS, bool FAST>
__global__ void __launch_bounds__(CFG::NT, fwd_min_blocks<CFG>())
render_fwd_batch_kernel(const __grid_constant__ FwdBatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FwdBatchSmem<CFG>& sm = *reinterpret_cast<FwdBatchSmem<CFG>*>(smem_raw);
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
    FwdTileOut o = a.out;
    o.tile_last = a.out.tile_last + vp.tile_base;
    o.n_contrib = a.out.n_contrib + vp.pix_base;
    o.color = a.out.color + 3 * (size_t)vp.pix_base;
    o.T = a.out.T + vp.pix_base;
    render_tile_fwd<CFG, NS, false, false, false, false, false, FAST>(vp, sm.c2w, tile_x, tile_y, a.ranges[item],
                                                                      a.vals, va, o, o.tile_last + local, sm.s,
                                                                      sm.red);
    __syncthreads();  // shared state (item, camera, staging) is free for the next tile
  }
}

// The same persistent form with two pixels per thread (svr_render_pair.cuh).
template <class CFG, int NS, bool FAST>
__global__ void __launch_bounds__(CFG::NT, pair_min_blocks<CFG>())
render_fwd_batch_pair_kernel(const __grid_constant__ FwdBatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FwdBatchSmem<CFG>& sm = *reinterpret_cast<FwdBatchSmem<CFG>*>(smem_raw);
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
    FwdTileOut o = a.out;
    o.tile_last = a.out.tile_last + vp.tile_base;
    o.n_contrib = a.out.n_contrib + vp.pix_base;
    o.color = a.out.color + 3 * (size_t)vp.pix_base;
    o.T = a.out.T + vp.pix_base;
    render_tile_fwd_pair<CFG, NS, FAST>(vp, sm.c2w, tile_x, tile_y, a.ranges[item], a.vals, va, o,
                                        o.tile_last + local, sm.s, sm.red);
    __syncthreads();
  }
}

#define SVR_FWD_DISPATCH(KERNEL, GRID, STREAM, ...)                                                   \
  do {                                                                                                \
    const int _ns = ns;                                                                               \
    const bool _d = depth, _t = dist, _n = normal, _m = maxw;                                         \
    auto _launch = [&](auto kfn) { kfn<<<GRID, PlainTile::NT, 0, STREAM>>>(__VA_ARGS__); };           \
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
                       const uint32_t* order, cudaStream_t stream) {
  FwdArgs args{vp, ranges, vals, va, out, order};
  const dim3 grid(vp.grid_x * vp.grid_y * kPlainSub);
  SVR_FWD_DISPATCH(render_fwd_kernel, grid, stream, args);
}

// Tile configurations with a two-pixels-per-thread variant.
bool batch_pair_supported(int tile, int stage) {
  return (tile == 8 && (stage == 32 || stage == 64)) || (tile == 16 && (stage == 128 || stage == 256));
}

// Batched tile configurations: (tile size, staging depth).
bool batch_tile_supported(int tile, int stage) {
  return (tile == 16 && (stage == 128 || stage == 256 || stage == 512)) ||
         (tile == 8 && (stage == 32 || stage == 64 || stage == 128)) || (tile == 32 && stage == 256);
}

template <class CFG>
static void set_fwd_pair_attrs() {
  const int smem = (int)sizeof(FwdBatchSmem<CFG>);
  cudaFuncSetAttribute(render_fwd_batch_pair_kernel<CFG, 1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(render_fwd_batch_pair_kernel<CFG, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(render_fwd_batch_pair_kernel<CFG, 3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(render_fwd_batch_pair_kernel<CFG, 1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(render_fwd_batch_pair_kernel<CFG, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  cudaFuncSetAttribute(render_fwd_batch_pair_kernel<CFG, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <class CFG, int NS>
static void set_fwd_batch_attr() {
  cudaFuncSetAttribute(render_fwd_batch_kernel<CFG, NS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(FwdBatchSmem<CFG>));
  cudaFuncSetAttribute(render_fwd_batch_kernel<CFG, NS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(FwdBatchSmem<CFG>));
}

template <class CFG>
static void set_fwd_batch_attrs() {
  set_fwd_batch_attr<CFG, 1>();
  set_fwd_batch_attr<CFG, 2>();
  set_fwd_batch_attr<CFG, 3>();
}

void ensure_fwd_batch_attributes() {
  static std::once_flag flags[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  std::call_once(flags[dev], [] {
    set_fwd_batch_attrs<TileCfg<16, 128>>();
    set_fwd_batch_attrs<TileCfg<16, 256>>();
    set_fwd_batch_attrs<TileCfg<16, 512>>();
    set_fwd_batch_attrs<TileCfg<8, 32>>();
    set_fwd_batch_attrs<TileCfg<8, 64>>();
    set_fwd_batch_attrs<TileCfg<8, 128>>();
    set_fwd_batch_attrs<TileCfg<32, 256>>();
    set_fwd_pair_attrs<PairCfg<8, 32>>();
    set_fwd_pair_attrs<PairCfg<8, 64>>();
    set_fwd_pair_attrs<PairCfg<16, 128>>();
    set_fwd_pair_attrs<PairCfg<16, 256>>();
  });
}

template <class CFG, bool FAST>
static void launch_fwd_batch_arith(const FwdBatchArgs& args, int ns, int ctas_per_sm, cudaStream_t stream) {
  const size_t smem = sizeof(FwdBatchSmem<CFG>);
  auto go = [&](auto kfn) {
    const int grid = persistent_grid((const void*)kfn, CFG::NT, smem, args.n_items, ctas_per_sm);
    kfn<<<grid, CFG::NT, smem, stream>>>(args);
  };
  if (ns == 1) go(render_fwd_batch_kernel<CFG, 1, FAST>);
  else if (ns == 2) go(render_fwd_batch_kernel<CFG, 2, FAST>);
  else go(render_fwd_batch_kernel<CFG, 3, FAST>);
}

template <class CFG, bool FAST>
static void launch_fwd_pair_arith(const FwdBatchArgs& args, int ns, int ctas_per_sm, cudaStream_t stream) {
  const size_t smem = sizeof(FwdBatchSmem<CFG>);
  auto go = [&](auto kfn) {
    const int grid = persistent_grid((const void*)kfn, CFG::NT, smem, args.n_items, ctas_per_sm);
    kfn<<<grid, CFG::NT, smem, stream>>>(args);
  };
  if (ns == 1) go(render_fwd_batch_pair_kernel<CFG, 1, FAST>);
  else if (ns == 2) go(render_fwd_batch_pair_kernel<CFG, 2, FAST>);
  else go(render_fwd_batch_pair_kernel<CFG, 3, FAST>);
}

template <class CFG>
static void launch_fwd_pair_cfg(const FwdBatchArgs& args, int ns, bool fast, int ctas_per_sm, cudaStream_t stream) {
  if (fast) launch_fwd_pair_arith<CFG, true>(args, ns, ctas_per_sm, stream);
  else launch_fwd_pair_arith<CFG, false>(args, ns, ctas_per_sm, stream);
}

template <class CFG>
static void launch_fwd_batch_cfg(const FwdBatchArgs& args, int ns, bool fast, int ctas_per_sm, cudaStream_t stream) {
  if (fast) launch_fwd_batch_arith<CFG, true>(args, ns, ctas_per_sm, stream);
  else launch_fwd_batch_arith<CFG, false>(args, ns, ctas_per_sm, stream);
}

void launch_render_fwd_batch(const ViewTable& views, int n_items, const uint2* ranges,
                             const uint32_t* vals, const VoxelArrays& va, int P, size_t rgb_view_stride,
                             const FwdTileOut& out, int ns, int tile, int stage, bool fast, int pair,
                             const uint32_t* order, uint32_t* counter, int ctas_per_sm, cudaStream_t stream) {
  if (n_items <= 0) return;
  ensure_fwd_batch_attributes();
  cudaMemsetAsync(counter, 0, sizeof(uint32_t), stream);
  const FwdBatchArgs args{views, n_items, ranges, vals, va, P, rgb_view_stride, out, order, counter};
  if (pair && batch_pair_supported(tile, stage)) {
    if (tile == 8 && stage == 32) launch_fwd_pair_cfg<PairCfg<8, 32>>(args, ns, fast, ctas_per_sm, stream);
    else if (tile == 8) launch_fwd_pair_cfg<PairCfg<8, 64>>(args, ns, fast, ctas_per_sm, stream);
    else if (stage == 128) launch_fwd_pair_cfg<PairCfg<16, 128>>(args, ns, fast, ctas_per_sm, stream);
    else launch_fwd_pair_cfg<PairCfg<16, 256>>(args, ns, fast, ctas_per_sm, stream);
    return;
  }
  if (tile == 8 && stage == 32) launch_fwd_batch_cfg<TileCfg<8, 32>>(args, ns, fast, ctas_per_sm, stream);
  else if (tile == 8 && stage == 128) launch_fwd_batch_cfg<TileCfg<8, 128>>(args, ns, fast, ctas_per_sm, stream);
  else if (tile == 8) launch_fwd_batch_cfg<TileCfg<8, 64>>(args, ns, fast, ctas_per_sm, stream);
  else if (tile == 32) launch_fwd_batch_cfg<TileCfg<32, 256>>(args, ns, fast, ctas_per_sm, stream);
  else if (stage == 128) launch_fwd_batch_cfg<TileCfg<16, 128>>(args, ns, fast, ctas_per_sm, stream);
  else if (stage == 512) launch_fwd_batch_cfg<TileCfg<16, 512>>(args, ns, fast, ctas_per_sm, stream);
  else launch_fwd_batch_cfg<TileCfg<16, 256>>(args, ns, fast, ctas_per_sm, stream);
}

}  // namespace svr
