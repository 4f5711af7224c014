// Binning of octrees 21 levels deep (the reference's new_cuda backend,
// backends/new_cuda/src/config.h:16,24-34 and forward.cu:660-752).
//
// The Morton rank then takes 3 * 21 = 63 bits, so a (tile, rank) key no
// longer fits in 64 bits; the reference sorts 128-bit keys
// (auxiliary.h:17-25,66-87).  Here the same order comes from two stable LSD
// radix sorts of 64-bit keys: first every instance by its rank, carrying its
// generation index, then the rank-sorted indices by their tile.  A stable
// sort by tile of a rank-sorted list is the lexicographic (tile, rank) order,
// and equal (tile, rank) pairs keep generation order -- exactly what one
// stable sort of the wide key gives.  The sorted values, the wide keys (as
// lo = tile << 63 | rank, hi = tile >> 1, the reference's SortKey128 halves)
// and the tile ranges are then written where the 16-level path leaves its
// own, so compositing and its backward read them unchanged.
#include "svr_common.cuh"
#include "svr_kernels.h"

namespace svr {

__host__ __device__ constexpr uint64_t octant_repeat_deep(uint64_t q) {
  uint64_t v = 0;
  for (int l = 0; l < kDeepLevels; ++l) v = (v << 3) | q;
  return v;
}

// One (rank, index) pair per instance in generation order (forward.cu:518-571
// of new_cuda, with the instance's own index as the carried value), plus the
// instance's rank, tile and sort value by index.
__global__ void __launch_bounds__(256)
duplicate_deep_kernel(const __grid_constant__ ViewParams vp, int P, const int64_t* __restrict__ octpaths,
                      const uint2* __restrict__ bboxes, const uint32_t* __restrict__ quads,
                      const uint32_t* __restrict__ ndup, const uint32_t* __restrict__ scan,
                      uint64_t* __restrict__ sort_keys, uint32_t* __restrict__ sort_idx,
                      uint64_t* __restrict__ rank_of, uint32_t* __restrict__ tile_of, uint32_t* __restrict__ val_of,
                      uint32_t cap, uint32_t* __restrict__ err) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= P) return;
  const uint32_t n = ndup[idx];
  if (n == 0) return;
  const uint32_t end = scan[idx];
  uint32_t off = end - n;
  if (end > cap) atomicOr(err, SVR_DEVERR_CAPACITY);
  const uint32_t wend = min(end, cap);
  if ((uint32_t)idx >= (1u << kVoxIdBits)) {
    atomicOr(err, SVR_DEVERR_VOXID);
    return;
  }
  int tx0, ty0, tx1, ty1;
  bbox_tile_rect(bboxes[idx], vp.grid_x, vp.grid_y, vp.tile_shift, tx0, ty0, tx1, ty1);
  const uint64_t path = (uint64_t)octpaths[idx];
  const uint32_t qb = quads[idx];
  for (uint32_t q = 0; q < 8; ++q) {
    if (!(qb & (1u << q))) continue;
    const uint64_t rank = path ^ octant_repeat_deep(q);
    const uint32_t val = make_sort_val((uint32_t)idx, q);
    for (int y = ty0; y <= ty1; ++y) {
      for (int x = tx0; x <= tx1; ++x) {
        if (off < wend) {
          sort_keys[off] = rank;
          sort_idx[off] = off;
          rank_of[off] = rank;
          tile_of[off] = (uint32_t)(y * vp.grid_x + x);
          val_of[off] = val;
        }
        ++off;
      }
    }
  }
  if (off != end) atomicOr(err, SVR_DEVERR_DUP_MISMATCH);
}

// The rank-sorted indices keyed by their tile, for the stable sort by tile.
__global__ void deep_tile_keys_kernel(uint32_t n, const uint32_t* __restrict__ d_n, const uint32_t* __restrict__ idx,
                                      const uint32_t* __restrict__ tile_of, uint64_t* __restrict__ keys,
                                      uint32_t* __restrict__ vals) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= min(n, *d_n)) return;
  const uint32_t k = idx[i];
  keys[i] = tile_of[k];
  vals[i] = k;
}

// Sorted values and wide keys from the final index order (may run in place
// over the index array: every thread reads its own slot before writing it).
__global__ void deep_finalize_kernel(uint32_t n, const uint32_t* __restrict__ d_n, const uint32_t* idx,
                                     const uint64_t* __restrict__ rank_of, const uint32_t* __restrict__ tile_of,
                                     const uint32_t* __restrict__ val_of, uint32_t* vals_out, uint64_t* keys_lo,
                                     uint64_t* __restrict__ keys_hi) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= min(n, *d_n)) return;
  const uint32_t k = idx[i];
  const uint64_t tile = tile_of[k];
  vals_out[i] = val_of[k];
  keys_lo[i] = (tile << kDeepRankBits) | rank_of[k];
  keys_hi[i] = tile >> (64 - kDeepRankBits);
}

void launch_binning_deep(const ViewParams& vp, int P, const int64_t* octpaths, const uint2* bboxes,
                         const uint32_t* quads, const uint32_t* ndup, const uint32_t* scan, const uint32_t* d_n,
                         uint32_t n, const DeepBinning& b, uint2* ranges, uint32_t* err, cudaStream_t stream) {
  if (P <= 0 || n == 0) return;
  const uint32_t n_tiles = (uint32_t)vp.grid_x * (uint32_t)vp.grid_y;
  duplicate_deep_kernel<<<(P + 255) / 256, 256, 0, stream>>>(vp, P, octpaths, bboxes, quads, ndup, scan, b.keys_a,
                                                            b.vals_a, b.rank_of, b.tile_of, b.val_of, n, err);
  // stable sort by rank (63 bits), then by tile
  uint64_t* k[2] = {b.keys_a, b.keys_b};
  uint32_t* v[2] = {b.vals_a, b.vals_b};
  const int r1 = launch_radix_sort(k[0], v[0], k[1], v[1], nullptr, d_n, n, kDeepRankBits, b.sort_temp, stream);
  const unsigned g = (n + 255) / 256;
  deep_tile_keys_kernel<<<g, 256, 0, stream>>>(n, d_n, v[r1], b.tile_of, k[1 - r1], v[1 - r1]);
  int tile_bits = 0;
  while (tile_bits < 32 && ((n_tiles - 1) >> tile_bits)) ++tile_bits;
  const int r2 = launch_radix_sort(k[1 - r1], v[1 - r1], k[r1], v[r1], nullptr, d_n, n, std::max(tile_bits, 1),
                                   b.sort_temp, stream);
  const int fin = r2 ? r1 : 1 - r1;  // the pair holding (tile, final index)
  launch_tile_ranges(k[fin], nullptr, d_n, n, 0, 0u, n_tiles, ranges, stream);
  deep_finalize_kernel<<<g, 256, 0, stream>>>(n, d_n, v[fin], b.rank_of, b.tile_of, b.val_of, b.vals_out,
                                              b.keys_lo, b.keys_hi);
}

}  // namespace svr
