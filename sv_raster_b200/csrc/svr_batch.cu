// Multi-view batched path: N views of one voxel set projected, binned,
// composited and back-propagated with one launch per stage over all views,
// without any host round trip (capturable in a CUDA graph).
//
// No reference counterpart: the reference renders one view per call and
// reads the instance count back to the host (forward.cu:601-734).  Per view,
// the results are those of the plain path:
//   - projection is project_voxel (preprocess.cu:24-132 arithmetic), fused
//     with the SH colour of each visible (voxel, view) (sh_compute.cu:54-106);
//   - instances of all views share one flat array, view-major, keyed
//     [tile | rank position]: the position of the instance's (voxel,
//     quadrant) pair in the ascending order of all 8P pairs' Morton ranks
//     (ties by voxel, then quadrant: the reference's generation order).  The
//     positions are view-independent, built once per plan by one radix sort,
//     and order instances exactly as the 48-bit ranks do, in ceil(log2 8P)
//     bits instead of 48.  The rank itself is compressed for the position
//     sort: with every voxel at octree level <= L < 16 its lowest 3*(16-L)
//     bits are the quadrant repeated, so (rank >> 3*(16-L)) << 3 | quadrant
//     orders pairs exactly as the full rank does;
//   - compositing / backward are the same per-tile device functions.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/svr_b200.h"
#include "svr_common.cuh"
#include "svr_kernels.h"
#include "svr_project.cuh"
#include "svr_render.cuh"
#include "svr_render_bwd.cuh"
#include "svr_render_fwd.cuh"
#include "svr_sh.cuh"

using namespace svr;

namespace svr {
// Instance keys: tile id above bit 32, rank position below.
constexpr int kPosShift = 32;
}  // namespace svr

namespace {
constexpr size_t kAlign = 256;
inline size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
}  // namespace

namespace svr {

struct GroupTable {
  int n;
  int v0[kMaxViews + 1];          // first view of each group (+ end)
  uint32_t tile_base[kMaxViews];  // first global tile of each group
};

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// One thread per voxel, looping over the views: the voxel's centre, size and
// SH coefficients are read once (the coefficients on its first visible view)
// and kept in registers, so each view costs the projection arithmetic and
// the per-(view, voxel) writes only.
template <int DEG, typename TS>
__global__ void __launch_bounds__(128)
project_sh_kernel(const __grid_constant__ ViewTable views, int P, const float* __restrict__ centers,
                  const float* __restrict__ lengths, const TS* __restrict__ sh0, const TS* __restrict__ shs, int M,
                  const int64_t* __restrict__ octpaths, int level_low_bits, int tight, uint32_t* __restrict__ ndup,
                  uint2* __restrict__ bboxes, uint32_t* __restrict__ quads, float* __restrict__ rgbs,
                  uint32_t* __restrict__ err) {
  __shared__ float s_m[kMaxViews][24];           // w2c (12) and c2w (12) of every view
  for (int t = threadIdx.x; t < views.n * 24; t += blockDim.x) {
    const int v = t / 24, k = t % 24;
    s_m[v][k] = k < 12 ? views.v[v].w2c[k] : views.v[v].c2w[k - 12];
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  // voxels deeper than the plan's max level would break the compressed ranks
  if (level_low_bits > 0 && ((uint64_t)octpaths[i] & ((1ull << level_low_bits) - 1ull)) != 0ull)
    atomicOr(err, SVR_DEVERR_LEVEL);
  const float cx = centers[3 * (size_t)i], cy = centers[3 * (size_t)i + 1], cz = centers[3 * (size_t)i + 2];
  const float len = lengths[i];
  // The rest coefficients are read per visible view through the cache
  // (holding 45 of them in registers across the views cost the kernel half
  // its occupancy).
  const TS* sh = shs + (size_t)i * (M - 1) * 3;
  float c0[3];
  bool loaded = false;
  for (int v = 0; v < views.n; ++v) {
    const size_t o = (size_t)v * P + i;
    const float* m = s_m[v];
    Projection pr = project_voxel(views.v[v], m, m + 12, cx, cy, cz, len);
    if (tight) tighten_bbox(views.v[v], pr);
    ndup[o] = pr.n;
    bboxes[o] = pr.bbox;
    quads[o] = pr.quads;
    if (pr.n == 0) continue;
    if (!loaded) {
#pragma unroll
      for (int c = 0; c < 3; ++c) c0[c] = ldf(sh0, 3 * (size_t)i + c);
      loaded = true;
    }
    // View-dependent colour of this visible voxel (sh_compute.cu:54-106).
    float dx = cx - m[12 + 3], dy = cy - m[12 + 7], dz = cz - m[12 + 11];
    const float rn = rnorm3df(dx, dy, dz);
    dx = dx * rn; dy = dy * rn; dz = dz * rn;
#pragma unroll
    for (int c = 0; c < 3; ++c) rgbs[3 * o + c] = sh_channel<DEG>(dx, dy, dz, c0[c], sh, c);
  }
}

// Instance segment [start, start + count) of each sort group, clamped to the
// capacity so that an overflowing step still stays inside the buffers.
__global__ void group_segments_kernel(const __grid_constant__ GroupTable gt, int P, const uint32_t* __restrict__ scan,
                                      uint32_t cap, uint32_t* __restrict__ segs) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= gt.n) return;
  const size_t v0 = gt.v0[g], v1 = gt.v0[g + 1];
  const uint32_t start = min(v0 == 0 ? 0u : scan[v0 * P - 1], cap);
  const uint32_t end = min(scan[v1 * P - 1], cap);
  segs[2 * g] = start;
  segs[2 * g + 1] = end - start;
}

// Position of the k-th (0-based) set bit of m (k < popc(m)).
__device__ __forceinline__ int nth_set_bit(uint32_t m, int k) {
  int pos = 0;
  int c = __popc(m & 0xFFFFu);
  if (k >= c) { k -= c; pos += 16; m >>= 16; }
  c = __popc(m & 0xFFu);
  if (k >= c) { k -= c; pos += 8; m >>= 8; }
  c = __popc(m & 0xFu);
  if (k >= c) { k -= c; pos += 4; m >>= 4; }
  c = __popc(m & 0x3u);
  if (k >= c) { k -= c; pos += 2; m >>= 2; }
  if (k >= (int)(m & 1u)) pos += 1;
  return pos;
}

// Duplication with the stores of a warp coalesced.  The instances of the
// warp's 32 consecutive (view, voxel) pairs form one contiguous run of the
// scan; the warp walks that run 32 instances at a time, each lane decoding
// its instance (owning voxel, then quadrant / tile row / tile column in the
// plain path's generation order: quadrants ascending, tiles row-major,
// forward.cu:540-562).  MODE selects what happens to the decoded instance:
//   kDupWrite   key and value at its own slot (generation order, for the
//               radix sort over the tile bits);
//   kDupCount   +1 on its tile's instance count (counts[global tile]);
//   kDupScatter key and value at the next free position of its tile's range
//               (ranges[t].y is the tile's cursor, starting at ranges[t].x).
// Count and scatter aggregate the lanes of a warp that hit the same tile
// (match.any) into one atomic.  Both skip exactly the instances whose
// generation slot is beyond the capacity, so every tile's cursor ends at the
// end of its range.  Positions inside a tile follow the atomics' order; the
// per-tile segment sort that follows orders them by their unique rank
// positions, so the final lists do not depend on it.
constexpr int kDupWrite = 0, kDupCount = 1, kDupScatter = 2;

template <int MODE>
__global__ void __launch_bounds__(256)
duplicate_batch_kernel(const __grid_constant__ ViewTable views, int P, const uint32_t* __restrict__ rank_pos,
                       const uint2* __restrict__ bboxes, const uint32_t* __restrict__ quads,
                       const uint32_t* __restrict__ ndup, const uint32_t* __restrict__ scan,
                       uint64_t* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t cap,
                       uint32_t* __restrict__ err, uint32_t* __restrict__ counts, uint2* __restrict__ ranges) {
  const int view = blockIdx.y;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool valid = idx < P;
  const size_t o = (size_t)view * P + (valid ? idx : 0);
  const ViewParams& vp = views.v[view];
  const uint32_t n = valid ? ndup[o] : 0u;
  const uint32_t end = valid ? scan[o] : 0u;
  if (n > 0 && end > cap) atomicOr(err, SVR_DEVERR_CAPACITY);
  int tx0 = 0, ty0 = 0, tx1 = 0, ty1 = 0;
  uint32_t qb = 0;
  if (n > 0) {
    bbox_tile_rect(bboxes[o], vp.grid_x, vp.grid_y, vp.tile_shift, tx0, ty0, tx1, ty1);
    qb = quads[o];
    const uint32_t tiles = (uint32_t)((tx1 - tx0 + 1) * (ty1 - ty0 + 1));
    if (tiles * (uint32_t)__popc(qb) != n) atomicOr(err, SVR_DEVERR_DUP_MISMATCH);
  }
  // exclusive scan of n over the warp; the run starts at the first lane's scan offset
  uint32_t incl = n;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += t;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  if (total == 0u) return;
  const uint32_t off = incl - n;
  const uint32_t run0 = __shfl_sync(0xffffffffu, end - n, 0) + 0u;  // lane 0's start (valid even if n == 0)
  const uint32_t w = (uint32_t)(tx1 - tx0 + 1);
  const uint32_t tiles = w * (uint32_t)(ty1 - ty0 + 1);
  for (uint32_t cb = 0; cb < total; cb += 32) {
    const uint32_t p = cb + lane;
    // owning lane: the largest s with off_s <= p (offsets are non-decreasing)
    int sl = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const uint32_t t = __shfl_sync(0xffffffffu, off, sl + step);
      if (t <= p) sl += step;
    }
    const uint32_t k = p - __shfl_sync(0xffffffffu, off, sl);
    const uint32_t s_tiles = __shfl_sync(0xffffffffu, tiles, sl);
    const uint32_t s_w = __shfl_sync(0xffffffffu, w, sl);
    const int s_tx0 = __shfl_sync(0xffffffffu, tx0, sl), s_ty0 = __shfl_sync(0xffffffffu, ty0, sl);
    const uint32_t s_qb = __shfl_sync(0xffffffffu, qb, sl);
    const uint32_t slot = run0 + p;
    const bool active = p < total && slot < cap;
    uint32_t q = 0, vid = 0, local = 0;
    if (active) {
      const uint32_t qi = k / s_tiles, rem = k - qi * s_tiles;
      const uint32_t ty = (uint32_t)s_ty0 + rem / s_w, tx = (uint32_t)s_tx0 + rem % s_w;
      q = (uint32_t)nth_set_bit(s_qb, (int)qi);
      vid = (uint32_t)(blockIdx.x * blockDim.x + (threadIdx.x & ~31) + sl);
      local = ty * (uint32_t)vp.grid_x + tx;
    }
    if (MODE == kDupWrite) {
      if (active) {
        keys[slot] = ((uint64_t)(vp.sort_tile_off + local) << kPosShift) | rank_pos[8 * (size_t)vid + q];
        vals[slot] = make_sort_val(vid, q);
      }
    } else {
      // global tile of the instance; inactive lanes share a value no tile has
      const uint32_t gtile = active ? vp.tile_base + local : 0xffffffffu;
      const uint32_t peers = __match_any_sync(0xffffffffu, gtile);
      const int leader = __ffs(peers) - 1;
      if (MODE == kDupCount) {
        if (active && lane == leader) atomicAdd(counts + gtile, (uint32_t)__popc(peers));
      } else {
        uint32_t base = 0;
        if (active && lane == leader) base = atomicAdd(&ranges[gtile].y, (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (active) {
          const uint32_t pos = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
          keys[pos] = ((uint64_t)(vp.sort_tile_off + local) << kPosShift) | rank_pos[8 * (size_t)vid + q];
          vals[pos] = make_sort_val(vid, q);
        }
      }
    }
  }
}

// Binned ranges: from each tile's instance count and its inclusive scan,
// ranges[t] = (start, start); the scatter pass advances .y to the end.  Empty
// tiles get (0, 0), as the radix path leaves them.
__global__ void bin_ranges_kernel(uint32_t n_tiles, const uint32_t* __restrict__ counts,
                                  const uint32_t* __restrict__ incl, uint2* __restrict__ ranges) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tiles) return;
  const uint32_t n = counts[t], start = n ? incl[t] - n : 0u;
  ranges[t] = make_uint2(start, start);
}

// Rank-position table, step 1: the (compressed) Morton rank of every
// (voxel, quadrant) pair, pair i = 8 * voxel + quadrant, and its index.
// Thread 0 stores the pair count the sort reads.
__global__ void rank_pos_keys_kernel(int P, const int64_t* __restrict__ octpaths, int rank_bits,
                                     uint64_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                     uint32_t* __restrict__ d_n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *d_n = (uint32_t)(8 * (size_t)P);
  if (i >= 8 * (size_t)P) return;
  const uint64_t path = (uint64_t)octpaths[i >> 3];
  const uint32_t q = (uint32_t)(i & 7);
  const int low = (rank_bits == kRankBits) ? 0 : kRankBits - (rank_bits - 3);  // 3*(16-L)
  const uint64_t full = order_rank(path, q);
  keys[i] = (low == 0) ? full : (((full >> low) << 3) | q);
  vals[i] = (uint32_t)i;
}

// Step 2: after a stable sort of the keys, position k holds pair vals[k].
__global__ void rank_pos_scatter_kernel(size_t n, const uint32_t* __restrict__ sorted_pairs,
                                        uint32_t* __restrict__ rank_pos) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) rank_pos[sorted_pairs[k]] = (uint32_t)k;
}

// dL/dSH of every voxel summed over views: sum_v basis(dir_v) * dL/drgb_v
// (sh_compute.cu:110-176 per view), and the subdivision priority summed over
// views (backward.cu:514).  Views where the voxel got no colour gradient are
// skipped.  Each CTA stages its voxels' 3 + 3*(M-1) outputs in shared
// memory and stores them as contiguous rows (the per-voxel rows of dsh0 and
// dshs are 12 B and 180 B long, too short for coalesced per-thread stores).
constexpr int kShBwThreads = 128;

template <int DEG>
__global__ void __launch_bounds__(kShBwThreads)
sh_bw_batch_kernel(const __grid_constant__ ViewTable views, int P, int M, const float* __restrict__ centers,
                   const float4* __restrict__ drgbs, float* __restrict__ dsh0, float* __restrict__ dshs,
                   float* __restrict__ subdiv) {
  constexpr int NB = (DEG + 1) * (DEG + 1) - 1;
  __shared__ float s_pos[kMaxViews][3];
  extern __shared__ __align__(16) float s_out[];  // [kShBwThreads][3 + 3 * (M - 1)] then written out
  for (int v = threadIdx.x; v < views.n; v += blockDim.x) {
    s_pos[v][0] = views.v[v].c2w[3];
    s_pos[v][1] = views.v[v].c2w[7];
    s_pos[v][2] = views.v[v].c2w[11];
  }
  __syncthreads();
  const int rest = 3 * (M - 1);
  const int i0 = blockIdx.x * kShBwThreads;
  const int i = i0 + threadIdx.x;
  float a0[3] = {0.f, 0.f, 0.f};
  float sub = 0.f;
  float acc[NB > 0 ? NB : 1][3];
#pragma unroll
  for (int k = 0; k < (NB > 0 ? NB : 1); ++k) acc[k][0] = acc[k][1] = acc[k][2] = 0.f;
  if (i < P) {
    const float cx = centers[3 * (size_t)i], cy = centers[3 * (size_t)i + 1], cz = centers[3 * (size_t)i + 2];
    for (int v = 0; v < views.n; ++v) {
      const float4 g = drgbs[(size_t)v * P + i];
      const float g0 = g.x, g1 = g.y, g2 = g.z;
      sub += g.w;
      if (g0 == 0.f && g1 == 0.f && g2 == 0.f) continue;
      float x = cx - s_pos[v][0], y = cy - s_pos[v][1], z = cz - s_pos[v][2];
      const float rn = rnorm3df(x, y, z);
      x = x * rn; y = y * rn; z = z * rn;
      float basis[15];
      sh_basis_rest<DEG>(x, y, z, basis);
      a0[0] += kC0 * g0; a0[1] += kC0 * g1; a0[2] += kC0 * g2;
#pragma unroll
      for (int k = 0; k < NB; ++k) {
        acc[k][0] += basis[k] * g0;
        acc[k][1] += basis[k] * g1;
        acc[k][2] += basis[k] * g2;
      }
    }
  }
  if (subdiv && i < P) subdiv[i] = sub;
  // stage: dsh0 rows first ([kShBwThreads][3]), then dshs rows ([kShBwThreads][rest])
  float* s0 = s_out;
  float* s1 = s_out + 3 * kShBwThreads;
  const int t = threadIdx.x;
  s0[3 * t + 0] = a0[0];
  s0[3 * t + 1] = a0[1];
  s0[3 * t + 2] = a0[2];
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    s1[t * rest + 3 * k + 0] = acc[k][0];
    s1[t * rest + 3 * k + 1] = acc[k][1];
    s1[t * rest + 3 * k + 2] = acc[k][2];
  }
  for (int k = 3 * NB; k < rest; ++k) s1[t * rest + k] = 0.f;  // coefficients above the degree
  __syncthreads();
  const int nv = min(kShBwThreads, P - i0);
  float* o0 = dsh0 + 3 * (size_t)i0;
  for (int e = t; e < 3 * nv; e += kShBwThreads) o0[e] = s0[e];
  if (rest > 0) {
    float* o1 = dshs + (size_t)rest * i0;
    for (int e = t; e < rest * nv; e += kShBwThreads) o1[e] = s1[e];
  }
}

inline int bit_width_u64(uint64_t n) {
  int b = 0;
  while (b < 64 && (n >> b)) ++b;
  return b;
}

}  // namespace svr

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
struct svr_batch_plan {
  ViewTable vt;
  GroupTable gt;
  int V;
  int64_t P;
  size_t cap;
  int n_samp;
  int rank_bits;  // compressed Morton rank width (position-table sort)
  int pos_bits;   // bits of a rank position (ceil(log2(8P)))
  int key_bits;   // widest group key (all groups sorted with this many passes)
  bool pos_ready;                 // rank-position table built for pos_paths
  const int64_t* pos_paths;
  int64_t total_tiles, total_pixels;
  // compositing schedule (svr_batch_plan_set_schedule)
  int order_flags;        // bit 0: forward tiles largest first, bit 1: backward (else tile order)
  int fwd_ctas_per_sm;    // resident CTAs per SM of the persistent launches (0 = as many as fit)
  int bwd_ctas_per_sm;
  int seg_small_n, seg_chunk;  // segment-sort buckets (svr_batch_plan_set_sort_buckets)
  int tile_size;               // compositing tile size (8, 16 or 32), fixed at creation
  int stage;                   // records staged per round (svr_batch_plan_set_staging)
  int stage_bwd;               // the backward's, when set apart (svr_batch_plan_set_backward_staging)
  int atomic_lanes;            // backward reduction threshold (svr_batch_plan_set_reduction)
  int exact;                   // compositing arithmetic (svr_batch_plan_set_arithmetic): 1 exact, 0 fast
  int pair;                    // two pixels per compositing thread (svr_batch_plan_set_pixels_per_thread)
  int pair_bwd;                // the backward's, when set apart (-1: as pair)
  int culling;                 // pixel bbox (svr_batch_plan_set_culling): -1 follows exact, 0 rounded, 1 tight
  int binning;                 // 1: counting sort by tile, 0: radix over the tile bits (svr_batch_plan_set_binning)
  // workspace layout (byte offsets)
  size_t o_header, o_ndup, o_scan, o_bbox, o_quad, o_scan_tmp, o_rgbs, o_drgbs;
  size_t o_ka, o_kb, o_va, o_vb, o_sort_tmp, o_ranges, o_tile_last, o_ncontrib;
  size_t o_okey, o_oval, o_order_fwd, o_order_bwd, o_order_tmp, o_pos;
  size_t bytes;
};

namespace {

struct BatchPtrs {
  uint32_t* header;
  uint32_t* ndup;
  uint32_t* scan;
  uint2* bbox;
  uint32_t* quad;
  void* scan_tmp;
  float* rgbs;
  float* drgbs;
  uint64_t *ka, *kb;
  uint32_t *va, *vb;
  void* sort_tmp;
  uint2* ranges;
  uint32_t* tile_last;
  uint32_t* ncontrib;
  uint64_t* okey;       // [2][T] order sort keys
  uint32_t* oval;       // [T] order sort input values
  uint32_t* order_fwd;  // [T]
  uint32_t* order_bwd;  // [T]
  void* order_tmp;
  uint32_t* rank_pos;   // [8P] position of (voxel, quadrant) in rank order
};

BatchPtrs ptrs(const svr_batch_plan* p, void* ws) {
  char* b = static_cast<char*>(ws);
  BatchPtrs q;
  q.header = reinterpret_cast<uint32_t*>(b + p->o_header);
  q.ndup = reinterpret_cast<uint32_t*>(b + p->o_ndup);
  q.scan = reinterpret_cast<uint32_t*>(b + p->o_scan);
  q.bbox = reinterpret_cast<uint2*>(b + p->o_bbox);
  q.quad = reinterpret_cast<uint32_t*>(b + p->o_quad);
  q.scan_tmp = b + p->o_scan_tmp;
  q.rgbs = reinterpret_cast<float*>(b + p->o_rgbs);
  q.drgbs = reinterpret_cast<float*>(b + p->o_drgbs);
  q.ka = reinterpret_cast<uint64_t*>(b + p->o_ka);
  q.kb = reinterpret_cast<uint64_t*>(b + p->o_kb);
  q.va = reinterpret_cast<uint32_t*>(b + p->o_va);
  q.vb = reinterpret_cast<uint32_t*>(b + p->o_vb);
  q.sort_tmp = b + p->o_sort_tmp;
  q.ranges = reinterpret_cast<uint2*>(b + p->o_ranges);
  q.tile_last = reinterpret_cast<uint32_t*>(b + p->o_tile_last);
  q.ncontrib = reinterpret_cast<uint32_t*>(b + p->o_ncontrib);
  q.okey = reinterpret_cast<uint64_t*>(b + p->o_okey);
  q.oval = reinterpret_cast<uint32_t*>(b + p->o_oval);
  q.order_fwd = reinterpret_cast<uint32_t*>(b + p->o_order_fwd);
  q.order_bwd = reinterpret_cast<uint32_t*>(b + p->o_order_bwd);
  q.order_tmp = b + p->o_order_tmp;
  q.rank_pos = reinterpret_cast<uint32_t*>(b + p->o_pos);
  return q;
}

// Header words: [0] instance count, [1] error word, [2] forward work counter,
// [3] backward work counter, [4] tile count read by the order sort, [5] pair
// count read by the rank-position sort, [6] binned instance count (counting
// sort by tile), [16..] group segments.
constexpr int kHeaderWords = 16 + 2 * kMaxViews;

// Longest-first work order of all tiles into `order` (see launch_tile_order).
void build_tile_order(const svr_batch_plan* p, const BatchPtrs& q, const uint32_t* tile_last, uint32_t* order,
                      cudaStream_t stream) {
  launch_tile_order(q.ranges, tile_last, (uint32_t)p->total_tiles, q.okey, q.oval, order, q.header + 4, q.order_tmp,
                    stream);
}

inline int check_last() { return cudaGetLastError() == cudaSuccess ? SVR_OK : SVR_ERR_CUDA; }

}  // namespace

extern "C" {

int svr_batch_plan_create(int n_views, const svr_camera* cams, int64_t P, int64_t capacity, int n_samp_per_vox,
                          int max_level, int tile_size, svr_batch_plan** out, size_t* workspace_bytes) {
  if (!out || !workspace_bytes || !cams || n_views < 1 || n_views > kMaxViews || P < 1 ||
      P >= (1ll << kVoxIdBits) || capacity < 0 || capacity > 0xffffffffll || n_samp_per_vox < 1 ||
      n_samp_per_vox > kMaxSamples || max_level < 1 || max_level > kMaxLevels ||
      !(tile_size == 8 || tile_size == 16 || tile_size == 32))
    return SVR_ERR_SHAPE;
  const int tile_shift = tile_size == 8 ? 3 : (tile_size == 16 ? 4 : 5);
  svr_batch_plan* p = new svr_batch_plan();
  memset(&p->vt, 0, sizeof(p->vt));
  p->tile_size = tile_size;
  p->stage = tile_size == 8 ? 64 : 256;
  p->stage_bwd = p->stage;
  p->V = n_views;
  p->P = P;
  p->cap = (size_t)capacity;
  p->n_samp = n_samp_per_vox;
  p->rank_bits = (max_level >= kMaxLevels) ? kRankBits : 3 * max_level + 3;
  p->pos_bits = bit_width_u64((uint64_t)(8 * P - 1));
  p->pos_ready = false;
  p->pos_paths = nullptr;
  p->vt.n = n_views;
  int64_t tiles = 0, pix = 0;
  for (int v = 0; v < n_views; ++v) {
    const svr_camera& c = cams[v];
    if (c.width <= 0 || c.height <= 0 || c.width >= 65536 || c.height >= 65536 || !c.w2c || !c.c2w) {
      delete p;
      return SVR_ERR_SHAPE;
    }
    ViewParams& vp = p->vt.v[v];
    vp.W = c.width;
    vp.H = c.height;
    vp.grid_x = (c.width + tile_size - 1) / tile_size;
    vp.grid_y = (c.height + tile_size - 1) / tile_size;
    vp.tile_shift = tile_shift;
    vp.tanfovx = c.tanfovx;
    vp.tanfovy = c.tanfovy;
    vp.cx = c.cx;
    vp.cy = c.cy;
    vp.focal_x = 0.5f * c.width / c.tanfovx;
    vp.focal_y = 0.5f * c.height / c.tanfovy;
    vp.near_plane = c.near_plane;
    vp.bg = c.bg_color;
    vp.w2c = c.w2c;
    vp.c2w = c.c2w;
    vp.tile_base = (uint32_t)tiles;
    vp.pix_base = (uint32_t)pix;
    tiles += (int64_t)vp.grid_x * vp.grid_y;
    pix += (int64_t)c.width * c.height;
  }
  if (pix > 0xffffffffll) {
    delete p;
    return SVR_ERR_SHAPE;
  }
  p->total_tiles = tiles;
  p->total_pixels = pix;
  // Greedy sort groups: consecutive views while the group's key fits 64 bits
  // (SVR_MAX_KEY_BITS lowers that limit, to exercise grouping in tests).
  int key_limit = 64;
  if (const char* e = getenv("SVR_MAX_KEY_BITS")) key_limit = std::max(1, std::min(64, atoi(e)));
  p->gt.n = 0;
  p->key_bits = 0;
  int v = 0;
  while (v < n_views) {
    const int g = p->gt.n++;
    p->gt.v0[g] = v;
    p->gt.tile_base[g] = p->vt.v[v].tile_base;
    uint64_t gt_tiles = 0;
    int kb = 0;
    while (v < n_views) {
      const uint64_t t2 = gt_tiles + (uint64_t)p->vt.v[v].grid_x * p->vt.v[v].grid_y;
      const int kb2 = kPosShift + bit_width_u64(t2);
      if (kb2 > key_limit && gt_tiles > 0) break;
      if (kb2 > 64) {  // a single view does not fit
        delete p;
        return SVR_ERR_KEYBITS;
      }
      p->vt.v[v].sort_group = g;
      p->vt.v[v].sort_tile_off = (uint32_t)gt_tiles;
      gt_tiles = t2;
      kb = kb2;
      ++v;
    }
    p->key_bits = std::max(p->key_bits, kb);
  }
  p->gt.v0[p->gt.n] = n_views;
  // workspace layout
  const size_t VP = (size_t)n_views * (size_t)P;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    off = align_up(off);
    const size_t r = off;
    off += bytes;
    return r;
  };
  p->o_header = take(kHeaderWords * sizeof(uint32_t));
  p->o_ndup = take(VP * 4);
  p->o_scan = take(VP * 4);
  p->o_bbox = take(VP * 8);
  p->o_quad = take(VP * 4);
  p->o_scan_tmp = take(scan_temp_bytes(std::max(VP, (size_t)tiles)));  // instance scan, then the tile-count scan
  p->o_rgbs = take(VP * 12);
  p->o_drgbs = take(VP * 16);  // [V,P,4]: dL/drgb (xyz) and the subdivision priority (w)
  // the instance arrays also serve the one-time sort of the 8P rank keys
  const size_t kv = std::max(p->cap, (size_t)(8 * P));
  p->o_ka = take(kv * 8);
  p->o_kb = take(kv * 8);
  p->o_va = take(kv * 4);
  p->o_vb = take(kv * 4);
  p->o_sort_tmp = take(std::max(sort_temp_bytes(kv), seg_sort_temp_bytes(p->cap, (int)tiles)));
  p->o_ranges = take((size_t)tiles * 8);
  p->o_tile_last = take((size_t)tiles * 4);
  p->o_ncontrib = take((size_t)pix * 4);
  p->o_okey = take((size_t)tiles * 16);
  p->o_oval = take((size_t)tiles * 4);
  p->o_order_fwd = take((size_t)tiles * 4);
  p->o_order_bwd = take((size_t)tiles * 4);
  p->o_order_tmp = take(sort_temp_bytes((size_t)tiles));
  p->o_pos = take((size_t)(8 * P) * 4);
  p->bytes = align_up(off) + kAlign;
  p->order_flags = 3;
  p->fwd_ctas_per_sm = 0;
  p->bwd_ctas_per_sm = 0;
  p->seg_small_n = 512;
  p->seg_chunk = 4096;
  p->atomic_lanes = 1;
  p->exact = 0;
  p->pair = 0;
  p->pair_bwd = -1;
  p->culling = -1;
  p->binning = 1;
  ensure_segsort_attributes();
  ensure_fwd_batch_attributes();
  ensure_bwd_batch_attributes();
  ensure_sort_attributes();
  *out = p;
  *workspace_bytes = p->bytes;
  return SVR_OK;
}

void svr_batch_plan_destroy(svr_batch_plan* plan) { delete plan; }

int svr_batch_plan_invalidate_geometry(svr_batch_plan* p) {
  if (!p) return SVR_ERR_SHAPE;
  p->pos_ready = false;
  return SVR_OK;
}

int svr_batch_plan_set_schedule(svr_batch_plan* p, int order_flags, int fwd_ctas_per_sm, int bwd_ctas_per_sm) {
  if (!p || order_flags < 0 || order_flags > 3 || fwd_ctas_per_sm < 0 || bwd_ctas_per_sm < 0 ||
      fwd_ctas_per_sm > 32 || bwd_ctas_per_sm > 32)
    return SVR_ERR_SHAPE;
  p->order_flags = order_flags;
  p->fwd_ctas_per_sm = fwd_ctas_per_sm;
  p->bwd_ctas_per_sm = bwd_ctas_per_sm;
  return SVR_OK;
}
int svr_batch_plan_set_staging(svr_batch_plan* p, int stage) {
  if (!p || !batch_tile_supported(p->tile_size, stage)) return SVR_ERR_SHAPE;
  p->stage = stage;
  p->stage_bwd = stage;
  return SVR_OK;
}

int svr_batch_plan_set_backward_staging(svr_batch_plan* p, int stage) {
  if (!p || !batch_tile_supported(p->tile_size, stage)) return SVR_ERR_SHAPE;
  p->stage_bwd = stage;
  return SVR_OK;
}

int svr_batch_plan_tile_size(const svr_batch_plan* p) { return p ? p->tile_size : 0; }

int svr_batch_plan_set_pixels_per_thread(svr_batch_plan* p, int pixels) {
  if (!p || (pixels != 1 && pixels != 2)) return SVR_ERR_SHAPE;
  p->pair = pixels == 2;
  return SVR_OK;
}

int svr_batch_plan_set_backward_pixels_per_thread(svr_batch_plan* p, int pixels) {
  if (!p || pixels < 0 || pixels > 2) return SVR_ERR_SHAPE;
  p->pair_bwd = pixels == 0 ? -1 : (pixels == 2);
  return SVR_OK;
}

int svr_batch_plan_set_arithmetic(svr_batch_plan* p, int exact) {
  if (!p || (exact != 0 && exact != 1)) return SVR_ERR_SHAPE;
  p->exact = exact;
  return SVR_OK;
}

int svr_batch_plan_set_culling(svr_batch_plan* p, int culling) {
  if (!p || culling < -1 || culling > 1) return SVR_ERR_SHAPE;
  p->culling = culling;
  return SVR_OK;
}

int svr_batch_plan_set_reduction(svr_batch_plan* p, int atomic_lanes) {
  if (!p || atomic_lanes < 1 || atomic_lanes > 32) return SVR_ERR_SHAPE;
  p->atomic_lanes = atomic_lanes;
  return SVR_OK;
}

int svr_batch_plan_set_binning(svr_batch_plan* p, int binning) {
  if (!p || (binning != 0 && binning != 1)) return SVR_ERR_SHAPE;
  p->binning = binning;
  return SVR_OK;
}

int svr_batch_plan_set_sort_buckets(svr_batch_plan* p, int small_n, int chunk) {
  if (!p || !seg_buckets_supported(small_n, chunk)) return SVR_ERR_SHAPE;
  p->seg_small_n = small_n;
  p->seg_chunk = chunk;
  return SVR_OK;
}

int64_t svr_batch_plan_pixels(const svr_batch_plan* p) { return p ? p->total_pixels : 0; }
int64_t svr_batch_plan_tiles(const svr_batch_plan* p) { return p ? p->total_tiles : 0; }
int svr_batch_plan_groups(const svr_batch_plan* p) { return p ? p->gt.n : 0; }

const uint32_t* svr_batch_count_ptr(const svr_batch_plan* p, const void* ws) {
  return reinterpret_cast<const uint32_t*>(static_cast<const char*>(ws) + p->o_header);
}
const uint64_t* svr_batch_bbox_ptr(const svr_batch_plan* p, const void* ws) {
  return reinterpret_cast<const uint64_t*>(static_cast<const char*>(ws) + p->o_bbox);
}

uint32_t* svr_batch_error_ptr(const svr_batch_plan* p, void* ws) {
  return reinterpret_cast<uint32_t*>(static_cast<char*>(ws) + p->o_header) + 1;
}

int svr_batch_arrays(const svr_batch_plan* p, const void* ws, const float** rgbs, const float** drgbs,
                     const uint64_t** ranges, const uint32_t** tile_last, const uint32_t** n_contrib,
                     const uint32_t** ndup, const uint32_t** sorted_vals) {
  if (!p || !ws) return SVR_ERR_SHAPE;
  BatchPtrs q = ptrs(p, const_cast<void*>(ws));
  if (rgbs) *rgbs = q.rgbs;
  if (drgbs) *drgbs = q.drgbs;
  if (ranges) *ranges = reinterpret_cast<const uint64_t*>(q.ranges);
  if (tile_last) *tile_last = q.tile_last;
  if (n_contrib) *n_contrib = q.ncontrib;
  if (ndup) *ndup = q.ndup;
  if (sorted_vals) *sorted_vals = q.vb;
  return SVR_OK;
}

int svr_batch_prepare(svr_batch_plan* p, void* ws, const int64_t* octree_paths, const float* vox_centers,
                      const float* vox_lengths, const void* sh0, const void* shs, int sh_bf16, int sh_degree, int M,
                      void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (!p || !ws || !octree_paths || !vox_centers || !vox_lengths || !sh0 || sh_degree < 0 || sh_degree > 3 ||
      M - 1 < (sh_degree + 1) * (sh_degree + 1) - 1 || (M > 1 && !shs))
    return SVR_ERR_SHAPE;
  BatchPtrs q = ptrs(p, ws);
  const int P = (int)p->P;
  const size_t VP = (size_t)p->V * p->P;
  cudaMemsetAsync(q.header, 0, kHeaderWords * sizeof(uint32_t), stream);
  const dim3 pgrid((P + 127) / 128);
  const int level_low = (p->rank_bits == kRankBits) ? 0 : kRankBits - (p->rank_bits - 3);  // 3*(16-L)
  const int tight = p->culling < 0 ? !p->exact : p->culling;
#define SVR_PROJ(D)                                                                                           \
  if (sh_bf16)                                                                                                \
    project_sh_kernel<D, __nv_bfloat16><<<pgrid, 128, 0, stream>>>(                                           \
        p->vt, P, vox_centers, vox_lengths, (const __nv_bfloat16*)sh0, (const __nv_bfloat16*)shs, M,         \
        octree_paths, level_low, tight, q.ndup, q.bbox, q.quad, q.rgbs, q.header + 1);                        \
  else                                                                                                        \
    project_sh_kernel<D, float><<<pgrid, 128, 0, stream>>>(p->vt, P, vox_centers, vox_lengths,               \
                                                           (const float*)sh0, (const float*)shs, M,          \
                                                           octree_paths, level_low, tight, q.ndup, q.bbox,   \
                                                           q.quad, q.rgbs, q.header + 1);
  const dim3 grid((P + 255) / 256, p->V);
  switch (sh_degree) {
    case 0: SVR_PROJ(0) break;
    case 1: SVR_PROJ(1) break;
    case 2: SVR_PROJ(2) break;
    default: SVR_PROJ(3) break;
  }
#undef SVR_PROJ
  launch_scan_inclusive(q.ndup, q.scan, VP, q.scan_tmp, q.header, (unsigned long long)p->cap, q.header + 1, stream);
  uint32_t* segs = q.header + 16;
  group_segments_kernel<<<1, 64, 0, stream>>>(p->gt, P, q.scan, (uint32_t)p->cap, segs);
  // the counting sort writes every tile's range itself; otherwise (radix
  // grouping, or no instance capacity yet) empty tiles keep (0, 0)
  if (!p->binning || p->cap == 0) cudaMemsetAsync(q.ranges, 0, (size_t)p->total_tiles * sizeof(uint2), stream);
  if (!p->pos_ready || p->pos_paths != octree_paths) {
    // Rank positions of all (voxel, quadrant) pairs: one stable radix sort of
    // the 8P compressed ranks in the (still free) instance arrays.
    const size_t n8 = 8 * (size_t)P;
    rank_pos_keys_kernel<<<(unsigned)((n8 + 255) / 256), 256, 0, stream>>>(P, octree_paths, p->rank_bits, q.ka, q.va,
                                                                          q.header + 5);
    const int in_b = launch_radix_sort(q.ka, q.va, q.kb, q.vb, nullptr, q.header + 5, (uint32_t)n8, p->rank_bits,
                                       q.sort_tmp, stream);
    rank_pos_scatter_kernel<<<(unsigned)((n8 + 255) / 256), 256, 0, stream>>>(n8, in_b ? q.vb : q.va, q.rank_pos);
    p->pos_ready = true;
    p->pos_paths = octree_paths;
  }
  if (p->cap > 0) {
    // Two-level sort: LSD radix passes over the tile bits only put every
    // tile's instances together in generation order (ending in ka/va) -- or,
    // with binning on, a counting sort by tile puts them together in no
    // particular order -- then one CTA per tile sorts its segment by the
    // rank-position bits into kb/vb.  Rank positions are unique inside a
    // tile, so either way the result is the order of one stable sort by the
    // full key.
    const bool odd = (sort_passes(p->key_bits - kPosShift) & 1) != 0;
    uint64_t* k0 = odd ? q.kb : q.ka;
    uint32_t* v0 = odd ? q.vb : q.va;
    uint64_t* k1 = odd ? q.ka : q.kb;
    uint32_t* v1 = odd ? q.va : q.vb;
    if (p->binning) {
      // Counting sort by tile instead: per-tile counts, their scan, then
      // every instance scattered into its tile's range (in ka/va directly).
      const uint32_t T = (uint32_t)p->total_tiles;
      cudaMemsetAsync(q.oval, 0, (size_t)T * sizeof(uint32_t), stream);
      duplicate_batch_kernel<kDupCount><<<grid, 256, 0, stream>>>(p->vt, P, q.rank_pos, q.bbox, q.quad, q.ndup,
                                                                  q.scan, q.ka, q.va, (uint32_t)p->cap, q.header + 1,
                                                                  q.oval, q.ranges);
      launch_scan_inclusive(q.oval, q.order_fwd, T, q.scan_tmp, q.header + 6, ~0ull, nullptr, stream);
      bin_ranges_kernel<<<(T + 255) / 256, 256, 0, stream>>>(T, q.oval, q.order_fwd, q.ranges);
      duplicate_batch_kernel<kDupScatter><<<grid, 256, 0, stream>>>(p->vt, P, q.rank_pos, q.bbox, q.quad, q.ndup,
                                                                    q.scan, q.ka, q.va, (uint32_t)p->cap,
                                                                    q.header + 1, q.oval, q.ranges);
    } else {
      duplicate_batch_kernel<kDupWrite><<<grid, 256, 0, stream>>>(p->vt, P, q.rank_pos, q.bbox, q.quad, q.ndup,
                                                                  q.scan, k0, v0, (uint32_t)p->cap, q.header + 1,
                                                                  nullptr, nullptr);
      for (int g = 0; g < p->gt.n; ++g) {
        launch_radix_sort(k0, v0, k1, v1, segs + 2 * g, segs + 2 * g + 1, (uint32_t)p->cap, p->key_bits,
                          q.sort_tmp, stream, kPosShift);
        const uint32_t g_tiles = (g + 1 < p->gt.n ? p->gt.tile_base[g + 1] : (uint32_t)p->total_tiles) -
                                 p->gt.tile_base[g];
        launch_tile_ranges(q.ka, segs + 2 * g, segs + 2 * g + 1, (uint32_t)p->cap, kPosShift, p->gt.tile_base[g],
                           g_tiles, q.ranges, stream);
      }
    }
    // the radix histograms in sort_tmp are dead here; the segment sort reuses it
    launch_tile_segment_sort(q.ranges, (int)p->total_tiles, q.ka, q.va, q.kb, q.vb, p->pos_bits, p->cap,
                             q.sort_tmp, stream, p->seg_small_n, p->seg_chunk);
  }
  return check_last();
}

// Compositing of all views with the densities either per voxel (geos) or
// as grid points read through the voxels' corner indices (va.key).
static int batch_render(svr_batch_plan* p, void* ws, VoxelArrays va, float* out_color, float* out_T,
                        cudaStream_t stream) {
  BatchPtrs q = ptrs(p, ws);
  va.bboxes = q.bbox;
  va.rgbs = q.rgbs;
  FwdTileOut out{q.tile_last, q.ncontrib, out_color, nullptr, nullptr, out_T, nullptr};
  const bool ordered = (p->order_flags & 1) != 0;
  if (ordered) build_tile_order(p, q, nullptr, q.order_fwd, stream);
  launch_render_fwd_batch(p->vt, (int)p->total_tiles, q.ranges, p->cap > 0 ? q.vb : nullptr, va, (int)p->P,
                          (size_t)p->P * 3, out, p->n_samp, p->tile_size, p->stage, !p->exact, p->pair,
                          ordered ? q.order_fwd : nullptr, q.header + 2, p->fwd_ctas_per_sm, stream);
  return check_last();
}

static int batch_backward(svr_batch_plan* p, void* ws, VoxelArrays va, const float* out_T, const float* dL_dcolor,
                          const float* dL_dT, BwdTileOut out, cudaStream_t stream) {
  BatchPtrs q = ptrs(p, ws);
  cudaMemsetAsync(q.drgbs, 0, (size_t)p->V * p->P * 16, stream);
  va.bboxes = q.bbox;
  va.rgbs = q.rgbs;
  BwdTileIn in{out_T, q.ncontrib, dL_dcolor, nullptr, nullptr, dL_dT, nullptr, nullptr, 0.f, 0.f, 0.f,
               p->atomic_lanes};
  out.dL_drgbs = q.drgbs;
  out.err = q.header + 1;
  const bool ordered = (p->order_flags & 2) != 0;
  if (ordered) build_tile_order(p, q, q.tile_last, q.order_bwd, stream);
  launch_render_bwd_batch(p->vt, (int)p->total_tiles, q.ranges, q.tile_last, p->cap > 0 ? q.vb : nullptr, va,
                          (int)p->P, (size_t)p->P * 3, (size_t)p->P * 4, in, out, p->n_samp, p->tile_size,
                          p->stage_bwd, !p->exact, p->pair_bwd < 0 ? p->pair : p->pair_bwd,
                          ordered ? q.order_bwd : nullptr, q.header + 3,
                          p->bwd_ctas_per_sm, stream);
  return check_last();
}

int svr_batch_render(svr_batch_plan* p, void* ws, const float* vox_centers, const float* vox_lengths,
                     const void* geos, int geos_bf16, float* out_color, float* out_T, void* stream_) {
  if (!p || !ws || !vox_centers || !vox_lengths || !geos || !out_color || !out_T) return SVR_ERR_SHAPE;
  if ((reinterpret_cast<uintptr_t>(geos) & 15u) != 0) return SVR_ERR_ALIGN;
  VoxelArrays va{nullptr, vox_centers, vox_lengths, geos_bf16 ? nullptr : (const float*)geos,
                 geos_bf16 ? (const __nv_bfloat16*)geos : nullptr, nullptr};
  return batch_render(p, ws, va, out_color, out_T, static_cast<cudaStream_t>(stream_));
}

int svr_batch_render_grid(svr_batch_plan* p, void* ws, const float* vox_centers, const float* vox_lengths,
                          const int64_t* vox_key, const void* grid, int grid_bf16, float* out_color, float* out_T,
                          void* stream_) {
  if (!p || !ws || !vox_centers || !vox_lengths || !vox_key || !grid || !out_color || !out_T) return SVR_ERR_SHAPE;
  VoxelArrays va{nullptr, vox_centers, vox_lengths, nullptr, nullptr, nullptr};
  va.key = vox_key;
  va.grid = grid_bf16 ? nullptr : (const float*)grid;
  va.grid_bf16 = grid_bf16 ? (const __nv_bfloat16*)grid : nullptr;
  return batch_render(p, ws, va, out_color, out_T, static_cast<cudaStream_t>(stream_));
}

int svr_batch_backward(svr_batch_plan* p, void* ws, const float* vox_centers, const float* vox_lengths,
                       const void* geos, int geos_bf16, const float* out_T, const float* dL_dcolor,
                       const float* dL_dT, float* dL_dgeos, void* stream_) {
  if (!p || !ws || !vox_centers || !vox_lengths || !geos || !out_T || !dL_dcolor || !dL_dT || !dL_dgeos)
    return SVR_ERR_SHAPE;
  if ((reinterpret_cast<uintptr_t>(geos) & 15u) != 0 || (reinterpret_cast<uintptr_t>(dL_dgeos) & 15u) != 0)
    return SVR_ERR_ALIGN;
  VoxelArrays va{nullptr, vox_centers, vox_lengths, geos_bf16 ? nullptr : (const float*)geos,
                 geos_bf16 ? (const __nv_bfloat16*)geos : nullptr, nullptr};
  BwdTileOut out{dL_dgeos, nullptr, nullptr, nullptr, 1};
  return batch_backward(p, ws, va, out_T, dL_dcolor, dL_dT, out, static_cast<cudaStream_t>(stream_));
}

int svr_batch_backward_grid(svr_batch_plan* p, void* ws, const float* vox_centers, const float* vox_lengths,
                            const int64_t* vox_key, const void* grid, int grid_bf16, const float* out_T,
                            const float* dL_dcolor, const float* dL_dT, float* dL_dgrid, void* stream_) {
  if (!p || !ws || !vox_centers || !vox_lengths || !vox_key || !grid || !out_T || !dL_dcolor || !dL_dT || !dL_dgrid)
    return SVR_ERR_SHAPE;
  VoxelArrays va{nullptr, vox_centers, vox_lengths, nullptr, nullptr, nullptr};
  va.key = vox_key;
  va.grid = grid_bf16 ? nullptr : (const float*)grid;
  va.grid_bf16 = grid_bf16 ? (const __nv_bfloat16*)grid : nullptr;
  BwdTileOut out{nullptr, nullptr, nullptr, nullptr, 0};
  out.key = vox_key;
  out.grid_grad = dL_dgrid;
  return batch_backward(p, ws, va, out_T, dL_dcolor, dL_dT, out, static_cast<cudaStream_t>(stream_));
}

int svr_batch_sh_backward(svr_batch_plan* p, void* ws, const float* vox_centers, int sh_degree, int M,
                          float* dL_dsh0, float* dL_dshs, float* subdiv, void* stream_) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  if (!p || !ws || !vox_centers || !dL_dsh0 || sh_degree < 0 || sh_degree > 3 ||
      M - 1 < (sh_degree + 1) * (sh_degree + 1) - 1 || (M > 1 && !dL_dshs))
    return SVR_ERR_SHAPE;
  BatchPtrs q = ptrs(p, ws);
  const int P = (int)p->P;
  const int g = (P + kShBwThreads - 1) / kShBwThreads;
  const size_t smem = (size_t)kShBwThreads * (3 + 3 * (M - 1)) * sizeof(float);
  if (smem > 48 * 1024) return SVR_ERR_SHAPE;  // M <= 32 coefficients per channel
  const float4* d4 = reinterpret_cast<const float4*>(q.drgbs);
  switch (sh_degree) {
    case 0: sh_bw_batch_kernel<0><<<g, kShBwThreads, smem, stream>>>(p->vt, P, M, vox_centers, d4, dL_dsh0, dL_dshs, subdiv); break;
    case 1: sh_bw_batch_kernel<1><<<g, kShBwThreads, smem, stream>>>(p->vt, P, M, vox_centers, d4, dL_dsh0, dL_dshs, subdiv); break;
    case 2: sh_bw_batch_kernel<2><<<g, kShBwThreads, smem, stream>>>(p->vt, P, M, vox_centers, d4, dL_dsh0, dL_dshs, subdiv); break;
    default: sh_bw_batch_kernel<3><<<g, kShBwThreads, smem, stream>>>(p->vt, P, M, vox_centers, d4, dL_dsh0, dL_dshs, subdiv); break;
  }
  return check_last();
}

}  // extern "C"
