// Per-tile segment sort: after a global sort by tile id only, every tile's
// instances are contiguous and still in generation order; this file then
// sorts each tile's segment by the Morton-rank bits of the key, stably.
//
// Together this yields exactly the order of one stable sort by the full
// [tile | rank] key (forward.cu:678-686): the tile passes keep generation
// order inside a tile, and every step below orders by rank with generation
// order breaking ties.  The batched path may group by tile with a counting
// sort instead, which leaves a tile's instances in no particular order; its
// keys (rank positions) are unique inside a tile, so the sorted result is the
// same.
//
// Tile sizes are heavy-tailed (in a dense 1080p scene the median tile holds a
// few hundred instances while a few percent of the tiles hold tens of
// thousands and most of all instances), so the work is split by size:
//
//   plan    one thread per tile writes a work list: segments of at most
//           small_n instances, and chunks of at most `chunk` instances of the
//           larger segments (chunk c of a segment starts at c * chunk);
//   small   one 128-thread CTA per small segment: LSD 8-bit passes in shared
//           memory, result to (kb, vb);
//   chunk   one 512-thread CTA per chunk: the same passes on up to `chunk`
//           items; a segment of one chunk is final (to kb, vb), otherwise the
//           sorted run is written back in place (ka, va);
//   merge   one CTA per run of a multi-run segment: an item's final place is
//           its index in its run plus, for every other run, the number of
//           that run's keys ordered before it (keys <= it for earlier runs,
//           < it for later ones, which keeps ties in generation order),
//           counted by a merge-path walk of the two runs in shared memory.
//
// Passes whose digit is the same for the whole segment move nothing and are
// skipped.  All grids are persistent (fixed size, looping over the device-side
// work list), so the sequence is capturable in a CUDA graph.
#include "svr_block.cuh"
#include "svr_common.cuh"
#include "svr_kernels.h"

#include <algorithm>
#include <mutex>

namespace svr {

// Segment-size buckets (chosen per plan; the defaults are 512 and 4096):
// segments of at most small_n instances go to the small kernel, longer ones
// are cut into runs of `chunk` instances.
constexpr int kSmallThreads = 128;
constexpr int kChunkThreads = 512;
constexpr int kMergeThreads = 512;
constexpr int kMinSmallN = 256;  // smallest supported small_n / chunk: they size the work lists
constexpr int kMinChunk = 2048;

bool seg_buckets_supported(int small_n, int chunk) {
  return (small_n == 256 || small_n == 512 || small_n == 1024) && (chunk == 2048 || chunk == 4096);
}

// Shared memory of an LSD sort of up to CAP keys of type KT by NT threads.
// The payload moved with each key is its 16-bit index in the input; values
// are gathered from global memory once, after the last pass.  KT is uint32_t
// when the sorted bits fit 32 (the batched path's rank positions; the tile
// bits above them are the same for the whole segment and are put back on the
// way out), uint64_t otherwise (the plain path's 48-bit ranks).
template <int NT, int CAP, typename KT>
struct SortSmem {
  static_assert(CAP <= 65536, "16-bit payload indices");
  KT k[2][CAP];
  uint16_t idx[2][CAP];
  uint32_t wcnt[NT / 32][256];  // per-warp digit counts, then per-warp exclusive prefixes
  uint32_t dstart[256];         // exclusive digit starts
  uint32_t scan_tmp[NT / 32 + 1];
};

// Sorts the n (<= CAP) keys in sm.k[0] stably by key bits [0, rank_bits),
// carrying their input indices (sm.idx[0] must hold 0..n-1), and returns the
// buffer index (0 or 1) holding the result.  Warp w owns the contiguous items
// [w * chunk, (w + 1) * chunk), so ranking warp by warp and digit by digit
// keeps equal digits in input order.
template <int NT, int CAP, typename KT>
__device__ int smem_lsd_sort(SortSmem<NT, CAP, KT>& sm, int n, int rank_bits) {
  constexpr int NW = NT / 32;
  constexpr int R = CAP / NT;                   // rounds of 32 items per warp at most
  constexpr int DPT = NT >= 256 ? 1 : 256 / NT;  // digits owned per thread (consecutive)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool owner = tid * DPT < 256;
  const uint32_t lt = lanemask_lt();
  const int chunk = ((n + NT - 1) / NT) * 32;  // items per warp, multiple of 32
  const int rounds = chunk / 32;
  int cur = 0;
  for (int shift = 0; shift < rank_bits; shift += 8) {
    for (int i = tid; i < NW * 256; i += NT) (&sm.wcnt[0][0])[i] = 0u;
    __syncthreads();
    uint32_t dig[R], rk[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (r < rounds) {
        const int i = warp * chunk + r * 32 + lane;
        const bool valid = i < n;
        const uint32_t d = valid ? ((uint32_t)(sm.k[cur][i] >> shift) & 0xFFu) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & lt);
        const uint32_t base = valid ? sm.wcnt[warp][d] : 0u;
        __syncwarp();
        if (valid && before == 0) sm.wcnt[warp][d] = base + __popc(peers);
        __syncwarp();
        dig[r] = d;
        rk[r] = base + before;
      }
    }
    __syncthreads();
    uint32_t tot_d[DPT], sum = 0;
    bool trivial = false;
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      tot_d[j] = 0;
      if (owner) {
        const int d = tid * DPT + j;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
          const uint32_t c = sm.wcnt[w][d];
          sm.wcnt[w][d] = run;
          run += c;
        }
        tot_d[j] = run;
        sum += run;
        trivial |= (run == (uint32_t)n);
      }
    }
    uint32_t all;
    uint32_t base = block_exclusive_scan<NT>(sum, sm.scan_tmp, all);
    if (owner) {
#pragma unroll
      for (int j = 0; j < DPT; ++j) {
        sm.dstart[tid * DPT + j] = base;
        base += tot_d[j];
      }
    }
    // one digit holds every key: nothing moves (block-uniform decision)
    if (__syncthreads_or(trivial)) continue;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (r < rounds) {
        const int i = warp * chunk + r * 32 + lane;
        if (i < n) {
          const uint32_t d = dig[r];
          const uint32_t pos = sm.dstart[d] + sm.wcnt[warp][d] + rk[r];
          sm.k[cur ^ 1][pos] = sm.k[cur][i];
          sm.idx[cur ^ 1][pos] = sm.idx[cur][i];
        }
      }
    }
    __syncthreads();
    cur ^= 1;
  }
  return cur;
}

// Work list: [0] small count, [1] chunk count, then the lists.
struct SegLists {
  uint32_t* counters;
  uint2* small;  // (start, n)
  uint4* chunk;  // (chunk start, chunk n, segment start, segment n)
  uint32_t small_cap, chunk_cap;
  uint32_t small_n, chunk_n;  // bucket limits of this launch
};

inline size_t seg_align(size_t x) { return (x + 255) / 256 * 256; }

// Chunk-list capacity for the smallest supported buckets (an upper bound for all).
inline uint32_t seg_chunk_cap(size_t cap, int n_tiles) {
  const size_t big_tiles = std::min<size_t>((size_t)n_tiles, cap / (kMinSmallN + 1));
  return (uint32_t)(cap / kMinChunk + big_tiles + 1);
}

size_t seg_sort_temp_bytes(size_t cap, int n_tiles) {
  return 256 + seg_align((size_t)n_tiles * sizeof(uint2)) + (size_t)seg_chunk_cap(cap, n_tiles) * sizeof(uint4);
}

static SegLists seg_lists(void* temp, size_t cap, int n_tiles, int small_n, int chunk) {
  char* b = static_cast<char*>(temp);
  SegLists L;
  L.small_n = (uint32_t)small_n;
  L.chunk_n = (uint32_t)chunk;
  L.counters = reinterpret_cast<uint32_t*>(b);
  L.small = reinterpret_cast<uint2*>(b + 256);
  L.chunk = reinterpret_cast<uint4*>(b + 256 + seg_align((size_t)n_tiles * sizeof(uint2)));
  L.small_cap = (uint32_t)n_tiles;
  L.chunk_cap = seg_chunk_cap(cap, n_tiles);
  return L;
}

__global__ void __launch_bounds__(256)
seg_plan_kernel(const uint2* __restrict__ ranges, int n_tiles, SegLists L) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  uint32_t start = 0, n = 0;
  if (t < n_tiles) {
    const uint2 r = ranges[t];
    start = r.x;
    n = r.y - r.x;
  }
  const bool small = n > 0 && n <= L.small_n;
  const uint32_t nch = n > L.small_n ? (n + L.chunk_n - 1) / L.chunk_n : 0u;
  // warp-aggregated reservations in both lists
  const uint32_t sball = __ballot_sync(0xffffffffu, small);
  uint32_t inc = nch;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  const uint32_t ctot = __shfl_sync(0xffffffffu, inc, 31);
  uint32_t sbase = 0, cbase = 0;
  if (lane == 0) {
    if (sball) sbase = atomicAdd(&L.counters[0], (uint32_t)__popc(sball));
    if (ctot) cbase = atomicAdd(&L.counters[1], ctot);
  }
  sbase = __shfl_sync(0xffffffffu, sbase, 0);
  cbase = __shfl_sync(0xffffffffu, cbase, 0);
  if (small) {
    const uint32_t s = sbase + __popc(sball & lanemask_lt());
    if (s < L.small_cap) L.small[s] = make_uint2(start, n);
  }
  for (uint32_t c = 0; c < nch; ++c) {
    const uint32_t e = cbase + inc - nch + c;
    if (e < L.chunk_cap) L.chunk[e] = make_uint4(start + c * L.chunk_n, min(L.chunk_n, n - c * L.chunk_n), start, n);
  }
}

// Key bits above a KT key: kept from the segment's first key (they are the
// same for the whole segment when KT is narrower than the key).
template <typename KT>
__device__ __forceinline__ uint64_t high_bits(uint64_t key) {
  return sizeof(KT) == 8 ? 0ull : (key & 0xFFFFFFFF00000000ull);
}

template <int SMALL_N, typename KT>
__global__ void __launch_bounds__(kSmallThreads)
seg_small_kernel(SegLists L, const uint64_t* __restrict__ ka, const uint32_t* __restrict__ va,
                 uint64_t* __restrict__ kb, uint32_t* __restrict__ vb, int rank_bits) {
  __shared__ SortSmem<kSmallThreads, SMALL_N, KT> sm;
  const uint32_t count = min(L.counters[0], L.small_cap);
  for (uint32_t e = blockIdx.x; e < count; e += gridDim.x) {
    const uint2 s = L.small[e];
    const int n = (int)s.y;
    const uint64_t hi = high_bits<KT>(ka[s.x]);
    __syncthreads();  // the previous segment's results have been read out
    for (int i = threadIdx.x; i < n; i += kSmallThreads) {
      sm.k[0][i] = (KT)ka[s.x + i];
      sm.idx[0][i] = (uint16_t)i;
    }
    __syncthreads();
    const int cur = smem_lsd_sort(sm, n, rank_bits);
    for (int i = threadIdx.x; i < n; i += kSmallThreads) {
      kb[s.x + i] = hi | (uint64_t)sm.k[cur][i];
      vb[s.x + i] = va[s.x + sm.idx[cur][i]];
    }
  }
}

template <int CHUNK, typename KT>
using ChunkSmem = SortSmem<kChunkThreads, CHUNK, KT>;

template <int CHUNK, typename KT>
__global__ void __launch_bounds__(kChunkThreads, 2)
seg_chunk_kernel(SegLists L, uint64_t* __restrict__ ka, uint32_t* __restrict__ va, uint64_t* __restrict__ kb,
                 uint32_t* __restrict__ vb, int rank_bits) {
  constexpr int kChunk = CHUNK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ChunkSmem<CHUNK, KT>& sm = *reinterpret_cast<ChunkSmem<CHUNK, KT>*>(smem_raw);
  const uint32_t count = min(L.counters[1], L.chunk_cap);
  for (uint32_t e = blockIdx.x; e < count; e += gridDim.x) {
    const uint4 c = L.chunk[e];
    const int n = (int)c.y;
    const uint64_t hi = high_bits<KT>(ka[c.x]);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kChunkThreads) {
      sm.k[0][i] = (KT)ka[c.x + i];
      sm.idx[0][i] = (uint16_t)i;
    }
    __syncthreads();
    const int cur = smem_lsd_sort(sm, n, rank_bits);
    if (c.w == c.y) {  // a single-chunk segment is final
      for (int i = threadIdx.x; i < n; i += kChunkThreads) {
        kb[c.x + i] = hi | (uint64_t)sm.k[cur][i];
        vb[c.x + i] = va[c.x + sm.idx[cur][i]];
      }
    } else {  // the sorted run goes back in place: gather every value before any is overwritten
      constexpr int kPer = kChunk / kChunkThreads;
      uint32_t vv[kPer];
#pragma unroll
      for (int j = 0; j < kPer; ++j) {
        const int i = threadIdx.x + j * kChunkThreads;
        vv[j] = i < n ? va[c.x + sm.idx[cur][i]] : 0u;
      }
      __syncthreads();
#pragma unroll
      for (int j = 0; j < kPer; ++j) {
        const int i = threadIdx.x + j * kChunkThreads;
        if (i < n) {
          ka[c.x + i] = hi | (uint64_t)sm.k[cur][i];
          va[c.x + i] = vv[j];
        }
      }
    }
  }
}

template <int CHUNK, typename KT>
struct MergeSmem {
  KT own[CHUNK];
  KT other[CHUNK];
  uint32_t cnt[CHUNK];  // per own item: keys of the other runs ordered before it
};

// Merge-path co-ranking of run `own` (index r) against run `other` (index
// s): thread t walks the merged order's outputs [t * per, (t + 1) * per) and,
// for every own item it passes, adds the number of other-run keys before it.
// On equal keys the earlier run comes first.
template <int CHUNK, typename KT>
__device__ __forceinline__ void corank_run(MergeSmem<CHUNK, KT>& sm, uint32_t n_own, uint32_t n_oth,
                                           bool own_first_on_tie) {
  const uint32_t total = n_own + n_oth;
  const uint32_t per = (total + kMergeThreads - 1) / kMergeThreads;
  const uint32_t d0 = min(total, threadIdx.x * per), d1 = min(total, d0 + per);
  if (d0 >= d1) return;
  // own[i] comes before other[j] in the merged order
  auto own_before = [&](KT a, KT b) { return own_first_on_tie ? (a <= b) : (a < b); };
  // i = number of own items among the first d0 outputs: the smallest i with
  // own[i] not before other[d0 - 1 - i]
  uint32_t lo = d0 > n_oth ? d0 - n_oth : 0u, hi = min(d0, n_own);
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (own_before(sm.own[mid], sm.other[d0 - 1 - mid])) lo = mid + 1;
    else hi = mid;
  }
  uint32_t i = lo, j = d0 - lo;
  for (uint32_t d = d0; d < d1; ++d) {
    if (i < n_own && (j >= n_oth || own_before(sm.own[i], sm.other[j]))) {
      sm.cnt[i] += j;
      ++i;
    } else {
      ++j;
    }
  }
}

template <int CHUNK, typename KT>
__global__ void __launch_bounds__(kMergeThreads)
seg_merge_kernel(SegLists L, const uint64_t* __restrict__ ka, const uint32_t* __restrict__ va,
                 uint64_t* __restrict__ kb, uint32_t* __restrict__ vb) {
  constexpr int kChunk = CHUNK;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  MergeSmem<CHUNK, KT>& sm = *reinterpret_cast<MergeSmem<CHUNK, KT>*>(smem_raw);
  const uint32_t count = min(L.counters[1], L.chunk_cap);
  const int tid = threadIdx.x;
  for (uint32_t e = blockIdx.x; e < count; e += gridDim.x) {
    const uint4 c = L.chunk[e];
    if (c.w == c.y) continue;  // single-chunk segment: already final (block-uniform)
    const uint32_t n = c.y, seg0 = c.z, seg_n = c.w;
    const uint32_t r = (c.x - seg0) / kChunk;
    const uint32_t runs = (seg_n + kChunk - 1) / kChunk;
    const uint64_t hi = high_bits<KT>(ka[seg0]);
    __syncthreads();
    for (uint32_t i = tid; i < n; i += kMergeThreads) {
      sm.own[i] = (KT)ka[c.x + i];
      sm.cnt[i] = 0u;
    }
    for (uint32_t s = 0; s < runs; ++s) {
      if (s == r) continue;
      const uint32_t s0 = seg0 + s * kChunk;
      const uint32_t ns = min((uint32_t)kChunk, seg_n - s * kChunk);
      __syncthreads();
      for (uint32_t i = tid; i < ns; i += kMergeThreads) sm.other[i] = (KT)ka[s0 + i];
      __syncthreads();
      corank_run(sm, n, ns, /*own_first_on_tie=*/r < s);
    }
    __syncthreads();
    for (uint32_t i = tid; i < n; i += kMergeThreads) {
      const uint32_t pos = i + sm.cnt[i];
      kb[seg0 + pos] = hi | (uint64_t)sm.own[i];
      vb[seg0 + pos] = va[c.x + i];
    }
  }
}

template <int CHUNK, typename KT>
static void set_chunk_merge_attrs() {
  cudaFuncSetAttribute(seg_chunk_kernel<CHUNK, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(ChunkSmem<CHUNK, KT>));
  cudaFuncSetAttribute(seg_merge_kernel<CHUNK, KT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(MergeSmem<CHUNK, KT>));
}

void ensure_segsort_attributes() {
  static std::once_flag flags[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  std::call_once(flags[dev], [] {
    set_chunk_merge_attrs<2048, uint64_t>();
    set_chunk_merge_attrs<4096, uint64_t>();
    set_chunk_merge_attrs<2048, uint32_t>();
    set_chunk_merge_attrs<4096, uint32_t>();
  });
}

static int sm_count() {
  int dev = 0, n = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

template <int CHUNK, typename KT>
static void launch_chunk_and_merge(const SegLists& L, int sms, uint64_t* ka, uint32_t* va, uint64_t* kb,
                                   uint32_t* vb, int rank_bits, cudaStream_t stream) {
  const int chunk_grid = (int)std::min<int64_t>(L.chunk_cap, (int64_t)sms * 2);
  seg_chunk_kernel<CHUNK, KT><<<chunk_grid, kChunkThreads, sizeof(ChunkSmem<CHUNK, KT>), stream>>>(L, ka, va, kb,
                                                                                                  vb, rank_bits);
  const int merge_grid = (int)std::min<int64_t>(L.chunk_cap, (int64_t)sms * 2);
  seg_merge_kernel<CHUNK, KT><<<merge_grid, kMergeThreads, sizeof(MergeSmem<CHUNK, KT>), stream>>>(L, ka, va, kb,
                                                                                                  vb);
}

template <typename KT>
static void launch_segments(const SegLists& L, int n_tiles, int small_n, int chunk, uint64_t* ka, uint32_t* va,
                            uint64_t* kb, uint32_t* vb, int rank_bits, cudaStream_t stream) {
  const int sms = sm_count();
  const int small_grid = (int)std::min<int64_t>(n_tiles, (int64_t)sms * 12);
  if (small_n == 256)
    seg_small_kernel<256, KT><<<small_grid, kSmallThreads, 0, stream>>>(L, ka, va, kb, vb, rank_bits);
  else if (small_n == 1024)
    seg_small_kernel<1024, KT><<<small_grid, kSmallThreads, 0, stream>>>(L, ka, va, kb, vb, rank_bits);
  else
    seg_small_kernel<512, KT><<<small_grid, kSmallThreads, 0, stream>>>(L, ka, va, kb, vb, rank_bits);
  if (chunk == 2048) launch_chunk_and_merge<2048, KT>(L, sms, ka, va, kb, vb, rank_bits, stream);
  else launch_chunk_and_merge<4096, KT>(L, sms, ka, va, kb, vb, rank_bits, stream);
}

void launch_tile_segment_sort(const uint2* ranges, int n_tiles, uint64_t* ka, uint32_t* va, uint64_t* kb,
                              uint32_t* vb, int rank_bits, size_t cap, void* temp, cudaStream_t stream,
                              int small_n, int chunk) {
  if (n_tiles <= 0 || cap == 0) return;
  if (!seg_buckets_supported(small_n, chunk)) {
    small_n = 512;
    chunk = 4096;
  }
  ensure_segsort_attributes();
  const SegLists L = seg_lists(temp, cap, n_tiles, small_n, chunk);
  cudaMemsetAsync(L.counters, 0, 2 * sizeof(uint32_t), stream);
  seg_plan_kernel<<<(n_tiles + 255) / 256, 256, 0, stream>>>(ranges, n_tiles, L);
  // keys whose sorted bits fit 32 are sorted as 32-bit words (the bits above
  // are the segment's tile, the same for all its keys)
  if (rank_bits <= 32) launch_segments<uint32_t>(L, n_tiles, small_n, chunk, ka, va, kb, vb, rank_bits, stream);
  else launch_segments<uint64_t>(L, n_tiles, small_n, chunk, ka, va, kb, vb, rank_bits, stream);
}

}  // namespace svr
