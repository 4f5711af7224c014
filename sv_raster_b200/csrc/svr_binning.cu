// Binning: inclusive scan of per-voxel duplicate counts, key/value
// duplication, a stable LSD radix sort of (tile | Morton rank) keys and the
// per-tile [start, end) ranges.
//
// Replaces, in forward.cu:601-700 of the reference backend, the CUB scan
// (forward.cu:643-648), the blocking count read-back (forward.cu:653), the
// duplicateWithKeys kernel (forward.cu:518-571), the CUB radix sort
// (forward.cu:681-686) and identifyTileRanges (forward.cu:576-598).
//
// Design: every kernel reads the instance count from device memory and is
// launched for a caller-given capacity, so the whole chain can be captured in
// a CUDA graph without a host round trip.  The sort is a three-kernel-per-pass
// LSD radix sort (upsweep histogram, per-digit row scan, stable downsweep)
// with 8- to 10-bit digits and 2048-item CTA tiles; ranks within a CTA come from
// warp __match_any_sync, which keeps it stable, so it reproduces the order of
// any other stable sort of the same keys.
#include "svr_common.cuh"
#include "svr_views.cuh"
#include "svr_kernels.h"
#include "svr_block.cuh"

#include <mutex>

namespace svr {

// --------------------------------------------------------------------------
// Inclusive scan of uint32 counts (three phases, no inter-CTA waiting)
// --------------------------------------------------------------------------
// kScanThreads, kScanItems and kScanTile are declared in svr_kernels.h.
size_t scan_temp_bytes(size_t n) {
  const size_t nb = (n + kScanTile - 1) / kScanTile;
  return (nb + 1) * sizeof(unsigned long long) + 256;
}

__global__ void __launch_bounds__(kScanThreads)
scan_reduce_kernel(const uint32_t* __restrict__ in, size_t n, unsigned long long* __restrict__ block_sums) {
  __shared__ unsigned long long s_warp[kScanThreads / 32 + 1];
  const size_t base = (size_t)blockIdx.x * kScanTile;
  unsigned long long s = 0;
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    const size_t i = base + (size_t)r * kScanThreads + threadIdx.x;
    if (i < n) s += in[i];
  }
  unsigned long long tot;
  block_exclusive_scan<kScanThreads>(s, s_warp, tot);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// Single CTA: exclusive scan of the block sums (in place); writes the grand
// total (clamped to 32 bits) and flags overflow of 32 bits or of `cap`.
__global__ void __launch_bounds__(1024)
scan_blocks_kernel(unsigned long long* __restrict__ block_sums, int nb, uint32_t* __restrict__ d_total,
                   unsigned long long cap, uint32_t* __restrict__ err) {
  __shared__ unsigned long long s_warp[1024 / 32 + 1];
  unsigned long long running = 0;
  for (int b0 = 0; b0 < nb; b0 += 1024) {
    const int i = b0 + threadIdx.x;
    const unsigned long long x = (i < nb) ? block_sums[i] : 0ull;
    unsigned long long tot;
    const unsigned long long ex = block_exclusive_scan<1024>(x, s_warp, tot);
    if (i < nb) block_sums[i] = running + ex;
    running += tot;
  }
  if (threadIdx.x == 0) {
    if (running > 0xffffffffull) {
      *d_total = 0xffffffffu;
      if (err) atomicOr(err, SVR_DEVERR_CAPACITY);
    } else {
      *d_total = (uint32_t)running;
      if (err && running > cap) atomicOr(err, SVR_DEVERR_CAPACITY);
    }
  }
}

__global__ void __launch_bounds__(kScanThreads)
scan_apply_kernel(const uint32_t* __restrict__ in, size_t n, const unsigned long long* __restrict__ block_off,
                  uint32_t* __restrict__ out) {
  __shared__ unsigned long long s_warp[kScanThreads / 32 + 1];
  // Each thread owns kScanItems consecutive items: load through shared memory
  // so global accesses stay coalesced.
  __shared__ uint32_t s_val[kScanTile];
  const size_t base = (size_t)blockIdx.x * kScanTile;
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    const int li = r * kScanThreads + threadIdx.x;
    const size_t i = base + li;
    s_val[li] = (i < n) ? in[i] : 0u;
  }
  __syncthreads();
  uint32_t v[kScanItems];
  unsigned long long s = 0;
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    v[r] = s_val[threadIdx.x * kScanItems + r];
    s += v[r];
  }
  unsigned long long tot;
  unsigned long long run = block_exclusive_scan<kScanThreads>(s, s_warp, tot) + block_off[blockIdx.x];
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    run += v[r];
    s_val[threadIdx.x * kScanItems + r] = (uint32_t)run;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kScanItems; ++r) {
    const int li = r * kScanThreads + threadIdx.x;
    const size_t i = base + li;
    if (i < n) out[i] = s_val[li];
  }
}

void launch_scan_inclusive(const uint32_t* in, uint32_t* out, size_t n, void* temp, uint32_t* d_total,
                           unsigned long long cap, uint32_t* err, cudaStream_t stream) {
  if (n == 0) {
    cudaMemsetAsync(d_total, 0, sizeof(uint32_t), stream);
    return;
  }
  const int nb = (int)((n + kScanTile - 1) / kScanTile);
  unsigned long long* sums = reinterpret_cast<unsigned long long*>(temp);
  scan_reduce_kernel<<<nb, kScanThreads, 0, stream>>>(in, n, sums);
  scan_blocks_kernel<<<1, 1024, 0, stream>>>(sums, nb, d_total, cap, err);
  scan_apply_kernel<<<nb, kScanThreads, 0, stream>>>(in, n, sums, out);
}

// --------------------------------------------------------------------------
// Duplication: one (key, value) per (voxel, camera quadrant, touched tile),
// emitted in quadrant-ascending, then row-major tile order at the voxel's
// scan offset (forward.cu:518-563).
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
duplicate_kernel(const __grid_constant__ ViewTable views, int P,
                 const int64_t* __restrict__ octpaths,
                 const uint2* __restrict__ bboxes, const uint32_t* __restrict__ quads,
                 const uint32_t* __restrict__ ndup, const uint32_t* __restrict__ scan,
                 uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                 uint32_t cap, uint32_t* __restrict__ err) {
  const int view = blockIdx.y;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= P) return;
  const size_t o = (size_t)view * P + idx;
  const uint32_t n = ndup[o];
  if (n == 0) return;
  const ViewParams& vp = views.v[view];
  const uint32_t end = scan[o];
  uint32_t off = end - n;
  // Past the capacity: flag it, and still write the instances that fit so
  // that every slot below the capacity holds a valid key.
  if (end > cap) atomicOr(err, SVR_DEVERR_CAPACITY);
  const uint32_t wend = min(end, cap);
  if ((uint32_t)idx >= (1u << kVoxIdBits)) {
    atomicOr(err, SVR_DEVERR_VOXID);
    return;
  }
  int tx0, ty0, tx1, ty1;
  bbox_tile_rect(bboxes[o], vp.grid_x, vp.grid_y, vp.tile_shift, tx0, ty0, tx1, ty1);
  const uint64_t path = (uint64_t)octpaths[idx];
  const uint32_t qb = quads[o];
  for (uint32_t q = 0; q < 8; ++q) {
    if (!(qb & (1u << q))) continue;
    const uint64_t rank = order_rank(path, q);
    const uint32_t val = make_sort_val((uint32_t)idx, q);
    for (int y = ty0; y <= ty1; ++y) {
      for (int x = tx0; x <= tx1; ++x) {
        const uint64_t tile = (uint64_t)(y * vp.grid_x + x);
        if (off < wend) {
          keys[off] = make_sort_key(tile, rank);
          vals[off] = val;
        }
        ++off;
      }
    }
  }
  if (off != end) atomicOr(err, SVR_DEVERR_DUP_MISMATCH);
}

void launch_duplicate(const ViewTable& views, int P, const int64_t* octpaths, const uint2* bboxes,
                      const uint32_t* quads, const uint32_t* ndup, const uint32_t* scan, uint64_t* keys,
                      uint32_t* vals, uint32_t cap, uint32_t* err, cudaStream_t stream) {
  if (P <= 0 || views.n <= 0) return;
  dim3 grid((P + 255) / 256, views.n);
  duplicate_kernel<<<grid, 256, 0, stream>>>(views, P, octpaths, bboxes, quads, ndup, scan, keys, vals, cap, err);
}

// --------------------------------------------------------------------------
// LSD radix sort of (uint64 key, uint32 value) pairs.  Digits are 8, 9 or 10
// bits wide: a sort over n key bits takes ceil(n / 10) passes of equal width
// (at least 8 bits), e.g. 2 passes of 9 bits for 18 bits instead of 3 of 8.
// --------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortRounds = 8;                        // items per thread (registers: keep >= 3 CTAs/SM)
constexpr int kSortTile = kSortThreads * kSortRounds;  // 2048
constexpr int kWarpSpan = 32 * kSortRounds;            // 256 items per warp
constexpr int kMaxRadixBits = 10;

static inline int sort_blocks(size_t cap) { return (int)((cap + kSortTile - 1) / kSortTile); }

size_t sort_temp_bytes(size_t cap) {
  const size_t nb = (size_t)std::max(1, sort_blocks(cap));
  const size_t radix = (size_t)1 << kMaxRadixBits;
  return (nb * radix + radix) * sizeof(uint32_t) + 256;
}

struct RadixPlan {
  int passes;
  int bits;  // digit width of every pass
};

static RadixPlan radix_plan(int nbits) {
  if (nbits <= 0) return {0, 8};
  const int passes = (nbits + kMaxRadixBits - 1) / kMaxRadixBits;
  const int bits = std::max(8, (nbits + passes - 1) / passes);
  return {passes, bits};
}

int sort_passes(int nbits) { return radix_plan(nbits).passes; }

template <int RB>
__global__ void __launch_bounds__(kSortThreads)
radix_upsweep_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ d_start,
                     const uint32_t* __restrict__ d_n, uint32_t cap, int shift, uint32_t* __restrict__ hist,
                     int nblocks) {
  constexpr int R = 1 << RB, DPT = R / kSortThreads;
  __shared__ uint32_t s_hist[kSortWarps][R];
  for (int i = threadIdx.x; i < kSortWarps * R; i += kSortThreads) (&s_hist[0][0])[i] = 0u;
  __syncthreads();
  const uint32_t n = min(*d_n, cap);
  if (d_start) keys += *d_start;
  const size_t start = (size_t)blockIdx.x * kSortTile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (start < n) {
#pragma unroll 4
    for (int r = 0; r < kSortRounds; ++r) {
      const size_t i = start + (size_t)warp * kWarpSpan + r * 32 + lane;
      if (i < n) {
        const uint32_t d = (uint32_t)(keys[i] >> shift) & (R - 1u);
        atomicAdd(&s_hist[warp][d], 1u);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < DPT; ++j) {
    const int d = threadIdx.x * DPT + j;
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) s += s_hist[w][d];
    hist[(size_t)d * nblocks + blockIdx.x] = s;
  }
}

// One CTA per digit: exclusive scan of that digit's per-block counts (in
// place) and the digit total.
__global__ void __launch_bounds__(1024)
radix_scan_rows_kernel(uint32_t* __restrict__ hist, int nblocks, uint32_t* __restrict__ digit_total) {
  __shared__ uint32_t s_warp[1024 / 32 + 1];
  uint32_t* row = hist + (size_t)blockIdx.x * nblocks;
  uint32_t running = 0;
  for (int b0 = 0; b0 < nblocks; b0 += 1024 * 4) {
    uint32_t v[4];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = b0 + threadIdx.x * 4 + k;
      v[k] = (i < nblocks) ? row[i] : 0u;
      s += v[k];
    }
    uint32_t tot;
    uint32_t ex = block_exclusive_scan<1024>(s, s_warp, tot) + running;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = b0 + threadIdx.x * 4 + k;
      if (i < nblocks) row[i] = ex;
      ex += v[k];
    }
    running += tot;
  }
  if (threadIdx.x == 0) digit_total[blockIdx.x] = running;
}

template <int RB>
struct DownsweepSmem {
  static constexpr int R = 1 << RB;
  uint64_t keys[kSortTile];
  uint32_t vals[kSortTile];
  uint32_t warp_cnt[kSortWarps][R];
  uint32_t local_start[R];
  uint32_t global_start[R];
  uint32_t scan_tmp[kSortThreads / 32 + 1];
};

template <int RB>
__global__ void __launch_bounds__(kSortThreads, 3)
radix_downsweep_kernel(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                       uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                       const uint32_t* __restrict__ d_start, const uint32_t* __restrict__ d_n, uint32_t cap, int shift,
                       const uint32_t* __restrict__ hist, const uint32_t* __restrict__ digit_total,
                       int nblocks) {
  constexpr int R = 1 << RB, DPT = R / kSortThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  DownsweepSmem<RB>& sm = *reinterpret_cast<DownsweepSmem<RB>*>(smem_raw);
  const uint32_t n = min(*d_n, cap);
  const size_t start = (size_t)blockIdx.x * kSortTile;
  if (start >= n) return;
  if (d_start) {
    const uint32_t s0 = *d_start;
    kin += s0; vin += s0; kout += s0; vout += s0;
  }
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (int i = tid; i < kSortWarps * R; i += kSortThreads) (&sm.warp_cnt[0][0])[i] = 0u;
  {
    // thread t owns digits [t * DPT, (t + 1) * DPT)
    uint32_t v[DPT], sum = 0;
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      v[j] = digit_total[tid * DPT + j];
      sum += v[j];
    }
    uint32_t tot;
    uint32_t gbase = block_exclusive_scan<kSortThreads>(sum, sm.scan_tmp, tot);
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      const int d = tid * DPT + j;
      sm.global_start[d] = gbase + hist[(size_t)d * nblocks + blockIdx.x];
      gbase += v[j];
    }
  }
  __syncthreads();

  uint64_t k[kSortRounds];
  uint32_t v[kSortRounds];
  uint32_t rk[kSortRounds];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const size_t i = start + (size_t)warp * kWarpSpan + r * 32 + lane;
    const bool valid = i < n;
    k[r] = valid ? kin[i] : 0ull;
    v[r] = valid ? vin[i] : 0u;
    const uint32_t d = valid ? ((uint32_t)(k[r] >> shift) & (R - 1u)) : (uint32_t)R;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t before = __popc(peers & lt);
    const uint32_t base = valid ? sm.warp_cnt[warp][d] : 0u;
    __syncwarp();
    if (valid && before == 0) sm.warp_cnt[warp][d] = base + __popc(peers);
    __syncwarp();
    rk[r] = base + before;
  }
  __syncthreads();
  {
    // Per digit: exclusive prefix over warps, then local start of the digit.
    uint32_t tot_d[DPT], sum = 0;
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      const int d = tid * DPT + j;
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = sm.warp_cnt[w][d];
        sm.warp_cnt[w][d] = run;
        run += c;
      }
      tot_d[j] = run;
      sum += run;
    }
    uint32_t tot;
    uint32_t base = block_exclusive_scan<kSortThreads>(sum, sm.scan_tmp, tot);
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
      sm.local_start[tid * DPT + j] = base;
      base += tot_d[j];
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const size_t i = start + (size_t)warp * kWarpSpan + r * 32 + lane;
    if (i < n) {
      const uint32_t d = (uint32_t)(k[r] >> shift) & (R - 1u);
      const uint32_t pos = sm.local_start[d] + sm.warp_cnt[warp][d] + rk[r];
      sm.keys[pos] = k[r];
      sm.vals[pos] = v[r];
    }
  }
  __syncthreads();
  const uint32_t tile_n = (uint32_t)min((size_t)kSortTile, (size_t)n - start);
  for (uint32_t p = tid; p < tile_n; p += kSortThreads) {
    const uint64_t key = sm.keys[p];
    const uint32_t d = (uint32_t)(key >> shift) & (R - 1u);
    const uint32_t g = sm.global_start[d] + (p - sm.local_start[d]);
    kout[g] = key;
    vout[g] = sm.vals[p];
  }
}

// Opt the downsweep kernels into >48 KB of dynamic shared memory, once per
// device (a function attribute, so it must not be set inside graph capture
// for the first time: plan creation and every plain call reach it first).
void ensure_sort_attributes() {
  static std::once_flag flags[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  std::call_once(flags[dev], [] {
    cudaFuncSetAttribute(radix_downsweep_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(DownsweepSmem<8>));
    cudaFuncSetAttribute(radix_downsweep_kernel<9>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(DownsweepSmem<9>));
    cudaFuncSetAttribute(radix_downsweep_kernel<10>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(DownsweepSmem<10>));
  });
}

template <int RB>
static void radix_pass(const uint64_t* kin, const uint32_t* vin, uint64_t* kout, uint32_t* vout,
                       const uint32_t* d_start, const uint32_t* d_n, uint32_t cap, int shift, uint32_t* hist,
                       uint32_t* digit_total, int nb, cudaStream_t stream) {
  radix_upsweep_kernel<RB><<<nb, kSortThreads, 0, stream>>>(kin, d_start, d_n, cap, shift, hist, nb);
  radix_scan_rows_kernel<<<1 << RB, 1024, 0, stream>>>(hist, nb, digit_total);
  radix_downsweep_kernel<RB><<<nb, kSortThreads, sizeof(DownsweepSmem<RB>), stream>>>(
      kin, vin, kout, vout, d_start, d_n, cap, shift, hist, digit_total, nb);
}

// Sorts the `*d_n` pairs starting at element `*d_start` (both read on the
// device; d_start may be null for 0) of (k0, v0) by key bits [lo_bit,
// key_bits), using (k1, v1) as the ping-pong buffer; `cap` bounds the count
// and sizes the grid.  Returns 0 if the result is in (k0, v0), 1 if in (k1, v1).
int launch_radix_sort(uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, const uint32_t* d_start,
                      const uint32_t* d_n, uint32_t cap, int key_bits, void* temp, cudaStream_t stream,
                      int lo_bit) {
  const RadixPlan rp = radix_plan(key_bits - lo_bit);
  if (cap == 0 || rp.passes == 0) return 0;
  const int nb = sort_blocks(cap);
  uint32_t* hist = reinterpret_cast<uint32_t*>(temp);
  uint32_t* digit_total = hist + (size_t)nb * (1u << rp.bits);
  ensure_sort_attributes();
  uint64_t* kin = k0; uint32_t* vin = v0; uint64_t* kout = k1; uint32_t* vout = v1;
  for (int p = 0; p < rp.passes; ++p) {
    const int shift = lo_bit + rp.bits * p;
    if (rp.bits == 8) radix_pass<8>(kin, vin, kout, vout, d_start, d_n, cap, shift, hist, digit_total, nb, stream);
    else if (rp.bits == 9) radix_pass<9>(kin, vin, kout, vout, d_start, d_n, cap, shift, hist, digit_total, nb, stream);
    else radix_pass<10>(kin, vin, kout, vout, d_start, d_n, cap, shift, hist, digit_total, nb, stream);
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  return rp.passes & 1;
}

// --------------------------------------------------------------------------
// Tile ranges from the sorted keys (forward.cu:576-598); `ranges` must be
// zeroed beforehand.  The segment [*d_start, *d_start + *d_n) holds keys
// whose bits above `rank_bits` are a tile id relative to `tile_base`; ranges
// are written as absolute element offsets.
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
tile_ranges_kernel(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ d_start,
                   const uint32_t* __restrict__ d_n, uint32_t cap, int rank_bits, uint32_t tile_base,
                   uint32_t n_tiles, uint2* __restrict__ ranges) {
  const uint32_t n = min(*d_n, cap);
  const uint32_t s0 = d_start ? *d_start : 0u;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys += s0;
  ranges += tile_base;
  const uint32_t cur = (uint32_t)(keys[i] >> rank_bits);
  const uint32_t prv = i > 0 ? (uint32_t)(keys[i - 1] >> rank_bits) : 0u;
  if (cur >= n_tiles || prv >= n_tiles) return;  // cannot happen for keys written by duplication
  if (i == 0) {
    ranges[cur].x = s0;
  } else {
    if (cur != prv) {
      ranges[prv].y = s0 + i;
      ranges[cur].x = s0 + i;
    }
  }
  if (i == n - 1) ranges[cur].y = s0 + n;
}

void launch_tile_ranges(const uint64_t* keys, const uint32_t* d_start, const uint32_t* d_n, uint32_t cap,
                        int rank_bits, uint32_t tile_base, uint32_t n_tiles, uint2* ranges, cudaStream_t stream) {
  if (cap == 0) return;
  tile_ranges_kernel<<<(cap + 255) / 256, 256, 0, stream>>>(keys, d_start, d_n, cap, rank_bits, tile_base, n_tiles,
                                                           ranges);
}

// --------------------------------------------------------------------------
// Tile work order for the compositing launches: tiles listed largest first
// by their instance count (eighth-octave buckets, tile order within a
// bucket).  Key = one 8-bit digit, 255 minus the bucket; a stable one-pass
// radix sort gives the order.  Thread 0 also stores the tile count the sort
// reads.
// --------------------------------------------------------------------------
__global__ void tile_order_keys_kernel(const uint2* __restrict__ ranges, const uint32_t* __restrict__ tile_last,
                                       uint32_t n_tiles, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                       uint32_t* __restrict__ d_n) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) *d_n = n_tiles;
  if (t >= n_tiles) return;
  const uint2 r = ranges[t];
  const uint32_t end = tile_last ? tile_last[t] : r.y;
  const uint32_t cost = end > r.x ? end - r.x : 0u;
  const uint32_t bucket = min(255u, (uint32_t)(log2f((float)cost + 1.f) * 7.9f));
  keys[t] = 255u - bucket;
  vals[t] = t;
}

size_t tile_order_temp_bytes(uint32_t n_tiles) { return sort_temp_bytes(n_tiles); }

void launch_tile_order(const uint2* ranges, const uint32_t* tile_last, uint32_t n_tiles, uint64_t* keys,
                       uint32_t* vals, uint32_t* order, uint32_t* d_n, void* temp, cudaStream_t stream) {
  if (n_tiles == 0) return;
  tile_order_keys_kernel<<<(n_tiles + 255) / 256, 256, 0, stream>>>(ranges, tile_last, n_tiles, keys, vals, d_n);
  launch_radix_sort(keys, vals, keys + n_tiles, order, nullptr, d_n, n_tiles, 8, temp, stream);
}

}  // namespace svr
