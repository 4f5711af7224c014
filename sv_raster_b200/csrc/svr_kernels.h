// Internal launcher declarations (host side of each kernel file).
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "svr_views.cuh"

namespace svr {

struct VoxelArrays;
struct FwdTileOut;
struct BwdTileIn;
struct BwdTileOut;

// svr_preprocess.cu
void launch_preprocess(const ViewTable& views, int P, const float* centers, const float* lengths, int32_t* out_ndup,
                       uint32_t* ndup, uint2* bboxes, uint32_t* quads, cudaStream_t stream);

// svr_binning.cu
// Inclusive scan: CTAs of kScanThreads threads, kScanItems items each; the
// scratch holds one 64-bit partial sum per CTA (scan_temp_bytes).
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;
size_t scan_temp_bytes(size_t n);
void launch_scan_inclusive(const uint32_t* in, uint32_t* out, size_t n, void* temp, uint32_t* d_total,
                           unsigned long long cap, uint32_t* err, cudaStream_t stream);
void launch_duplicate(const ViewTable& views, int P, const int64_t* octpaths, const uint2* bboxes,
                      const uint32_t* quads, const uint32_t* ndup, const uint32_t* scan, uint64_t* keys,
                      uint32_t* vals, uint32_t cap, uint32_t* err, cudaStream_t stream);
size_t sort_temp_bytes(size_t cap);
void ensure_sort_attributes();
int sort_passes(int key_bits);
int launch_radix_sort(uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, const uint32_t* d_start,
                      const uint32_t* d_n, uint32_t cap, int key_bits, void* temp, cudaStream_t stream,
                      int lo_bit = 0);
// Stable sort of every tile's segment [ranges[t].x, ranges[t].y) by the key
// bits below `rank_bits`, from (ka, va) into (kb, vb) (svr_segsort.cu).
// Sorts every tile's segment [ranges[t].x, ranges[t].y) of (ka, va) by key
// bits [0, rank_bits), stably, into the same positions of (kb, vb); ka/va are
// clobbered.  `cap` bounds the total instance count; temp holds
// seg_sort_temp_bytes(cap, n_tiles) bytes.
// small_n / chunk are the segment-size buckets (256|512|1024 and 2048|4096;
// other values fall back to 512 / 4096).
size_t seg_sort_temp_bytes(size_t cap, int n_tiles);
bool seg_buckets_supported(int small_n, int chunk);
void ensure_segsort_attributes();
void launch_tile_segment_sort(const uint2* ranges, int n_tiles, uint64_t* ka, uint32_t* va, uint64_t* kb,
                              uint32_t* vb, int rank_bits, size_t cap, void* temp, cudaStream_t stream,
                              int small_n = 512, int chunk = 4096);
// Largest-first work order of n_tiles tiles by instance count (cost =
// tile_last - start when tile_last is given, else the range length) into
// order[n_tiles]; keys [2 * n_tiles] and vals [n_tiles] are scratch, d_n one
// device word, temp tile_order_temp_bytes(n_tiles) bytes.
size_t tile_order_temp_bytes(uint32_t n_tiles);
void launch_tile_order(const uint2* ranges, const uint32_t* tile_last, uint32_t n_tiles, uint64_t* keys,
                       uint32_t* vals, uint32_t* order, uint32_t* d_n, void* temp, cudaStream_t stream);
void launch_tile_ranges(const uint64_t* keys, const uint32_t* d_start, const uint32_t* d_n, uint32_t cap,
                        int rank_bits, uint32_t tile_base, uint32_t n_tiles, uint2* ranges, cudaStream_t stream);

// svr_render_fwd.cu / svr_render_bwd.cu
// Plain one-view launches over the reference's 16x16 tile lists: four 8x8
// CTAs per list; CTA i renders quadrant i % 4 of list order[i / 4] (largest
// tiles first) or of list i / 4 when order is null.  The forward combines
// tile_last with atomicMax (the caller zeroes it).
void launch_render_fwd(const ViewParams& vp, const uint2* ranges, const uint32_t* vals, const VoxelArrays& va,
                       const FwdTileOut& out, int ns, bool depth, bool dist, bool normal, bool maxw,
                       const uint32_t* order, cudaStream_t stream);
// Multi-view forms (no depth / distortion / normal outputs): persistent
// grids taking tiles from `counter` (zeroed here) in the order of `order`
// (identity when null); ctas_per_sm caps the resident CTAs per SM (0 = as
// many as fit).  (tile, stage) must satisfy batch_tile_supported.
bool batch_pair_supported(int tile, int stage);
bool batch_tile_supported(int tile, int stage);
void ensure_fwd_batch_attributes();
void ensure_bwd_batch_attributes();
void launch_render_fwd_batch(const ViewTable& views, int n_items, const uint2* ranges,
                             const uint32_t* vals, const VoxelArrays& va, int P, size_t rgb_view_stride,
                             const FwdTileOut& out, int ns, int tile, int stage, bool fast, int pair,
                             const uint32_t* order, uint32_t* counter, int ctas_per_sm, cudaStream_t stream);
void launch_render_bwd(const ViewParams& vp, const uint2* ranges, const uint32_t* tile_last, const uint32_t* vals,
                       const VoxelArrays& va, const BwdTileIn& in, const BwdTileOut& out, int ns, bool depth,
                       bool dist, bool normal, const uint32_t* order, cudaStream_t stream);
void launch_render_bwd_batch(const ViewTable& views, int n_items, const uint2* ranges,
                             const uint32_t* tile_last, const uint32_t* vals, const VoxelArrays& va, int P,
                             size_t rgb_view_stride, size_t drgb_view_stride, const BwdTileIn& in,
                             const BwdTileOut& out, int ns, int tile, int stage, bool fast, int pair,
                             const uint32_t* order, uint32_t* counter, int ctas_per_sm, cudaStream_t stream);
// svr_binning_deep.cu: binning of 21-level octrees (63-bit ranks).  The
// sort pairs (keys_a, vals_a) / (keys_b, vals_b) and sort_temp are those of
// the 16-level layout; vals_out / keys_lo are its sorted-value and sorted-key
// arrays, keys_hi and the per-instance rank / tile / value arrays follow it.
struct DeepBinning {
  uint64_t* keys_a;
  uint64_t* keys_b;
  uint32_t* vals_a;
  uint32_t* vals_b;
  void* sort_temp;
  uint64_t* rank_of;
  uint32_t* tile_of;
  uint32_t* val_of;
  uint32_t* vals_out;
  uint64_t* keys_lo;
  uint64_t* keys_hi;
};
void launch_binning_deep(const ViewParams& vp, int P, const int64_t* octpaths, const uint2* bboxes,
                         const uint32_t* quads, const uint32_t* ndup, const uint32_t* scan, const uint32_t* d_n,
                         uint32_t n, const DeepBinning& b, uint2* ranges, uint32_t* err, cudaStream_t stream);
// Grid of a persistent launch: resident CTAs of `kernel` on this device
// (capped at ctas_per_sm per SM when > 0), at most n_items.
int persistent_grid(const void* kernel, int threads, size_t dyn_smem, int n_items, int ctas_per_sm);

// svr_sh_adam.cu
void launch_sh_eval(int deg, int n_idx, int P, int M, const int64_t* idx, const float* centers, const float* cam_pos,
                    const void* sh0, const void* shs, bool bf16, float* rgbs, cudaStream_t stream);
void launch_sh_eval_bw(int deg, int n_idx, int P, int M, const int64_t* idx, const float* centers,
                       const float* cam_pos, const float* dL_drgbs, float* dL_dsh0, float* dL_dshs,
                       cudaStream_t stream);
void launch_adam(bool biased, bool sparse, int64_t numel, float* param, const float* grad, float* m, float* v,
                 float step_or_lr, float beta1, float beta2, float rsqrt_bc2, float eps, cudaStream_t stream);

constexpr int kMaxAdamGroups = 8;
struct AdamGroup {
  void* param;         // fp32 or bf16
  const float* grad;
  float* exp_avg;
  float* exp_avg_sq;
  int64_t numel;
  float step_size, beta1, beta2, rsqrt_bc2, eps;
  int param_bf16;
  double lr;           // used with a device step counter
};
struct AdamGroupTable {
  int n;
  int sparse;
  const int* d_step;   // optional device step counter (bias correction on the device)
  double beta1d, beta2d;
  AdamGroup g[kMaxAdamGroups];
};
void launch_step_increment(int* d_step, cudaStream_t stream);
void launch_adam_fused(const AdamGroupTable& t, int num_sms, cudaStream_t stream);

void launch_gather(int dim, int n_care, const int64_t* vox_key, const int64_t* care_idx, const float* grid_pts,
                   float* out, cudaStream_t stream);
void launch_gather_bw(int dim, int n_care, const int64_t* vox_key, const int64_t* care_idx, const float* dL_dvox,
                      float* dL_dgrid, cudaStream_t stream);
// All voxels (no care list): corner densities from the grid (fp32 or bf16 in,
// fp32 or bf16 rows out), and the density gradients added into the grid's.
void launch_gather_all_geo(int64_t P, const int64_t* vox_key, const void* grid_pts, bool grid_bf16, void* out,
                           bool out_bf16, cudaStream_t stream);
void launch_scatter_all_geo(int64_t P, const int64_t* vox_key, const float* dL_dgeos, float* dL_dgrid,
                            cudaStream_t stream);

// svr_tv.cu
void launch_total_variation_bw(const float* grid, const int64_t* vox_key, float weight, const float* vox_size_inv,
                               bool no_tv_s, uint8_t* active, int64_t N, int C, float* grad, cudaStream_t stream);

}  // namespace svr
