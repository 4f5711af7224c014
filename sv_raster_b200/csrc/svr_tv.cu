// Total-variation gradient on the grid-point parameters: for every voxel and
// channel, each of its 8 corners gets weight * (sum over its 3 edge neighbours
// inside the voxel of sign(v_corner - v_neighbour)), optionally scaled by
// 0.01 / voxel size, added into the existing gradient
// (total_variation_bw_cuda, backends/cuda/src/tv_compute.cu:22-80).
//
// The "sparse" mode only touches voxels with a non-zero gradient on one of
// their corners.  The reference reads that gradient while other threads are
// already adding to it, so its result depends on scheduling; here the test
// reads the gradient as it was before this call (a first pass records it),
// which is the deterministic form of the same rule.
#include <type_traits>

#include "svr_common.cuh"
#include "svr_kernels.h"

namespace svr {

// One slot per (voxel, channel, corner), t = (n * C + c) * 8 + corner: the 8
// slots of a voxel-channel pair sit in an aligned group of 8 lanes, read the
// voxel's 8 keys as one contiguous run and exchange their corner values by
// shuffles (the edge neighbours of corner i inside the voxel are corners i^1,
// i^2 and i^4).  Each thread carries kTvSlots slots, 256 apart (so a lane keeps
// its corner), through every load stage together so their scattered reads
// are in flight at once.  No lane returns before the shuffles: warps are whole.
constexpr int kTvThreads = 256;
constexpr int kTvSlots = 4;

// CC > 0 fixes the channel count at compile time (no 64-bit division for the
// common one-channel grid); CC == 0 reads it from C.
template <int CC>
__global__ void __launch_bounds__(kTvThreads)
tv_active_kernel(int64_t n_slots, int C, const int64_t* __restrict__ vox_key, const float* __restrict__ grad,
                 uint8_t* __restrict__ active) {
  const int64_t base = (int64_t)blockIdx.x * (kTvThreads * kTvSlots) + threadIdx.x;
  const int lane = threadIdx.x & 31;
  if (CC > 0) C = CC;
  int64_t at[kTvSlots];
#pragma unroll
  for (int j = 0; j < kTvSlots; ++j) {
    const int64_t t = base + j * kTvThreads, nc = t >> 3;
    at[j] = t < n_slots ? vox_key[8 * (nc / C) + (t & 7)] * C + nc % C : -1;
  }
#pragma unroll
  for (int j = 0; j < kTvSlots; ++j) {
    const int64_t t = base + j * kTvThreads;
    const bool nz = at[j] >= 0 && grad[at[j]] != 0.f;
    const unsigned ball = __ballot_sync(0xffffffffu, nz);
    if (t < n_slots && (lane & 7) == 0) active[t >> 3] = ((ball >> lane) & 0xffu) != 0u;
  }
}

template <bool SCALE, int CC>
__global__ void __launch_bounds__(kTvThreads)
tv_grad_kernel(int64_t n_slots, int C, const float* __restrict__ grid, const int64_t* __restrict__ vox_key,
               float weight, const float* __restrict__ vox_size_inv, const uint8_t* __restrict__ active,
               float* __restrict__ grad) {
  const int64_t base = (int64_t)blockIdx.x * (kTvThreads * kTvSlots) + threadIdx.x;
  if (CC > 0) C = CC;
  int64_t at[kTvSlots];
  float v[kTvSlots], w[kTvSlots];
#pragma unroll
  for (int j = 0; j < kTvSlots; ++j) {
    const int64_t t = base + j * kTvThreads, nc = t >> 3;
    const bool on = t < n_slots && (!active || active[nc]);  // uniform over the 8 lanes of a group
    at[j] = on ? vox_key[8 * (nc / C) + (t & 7)] * C + nc % C : -1;
    w[j] = weight;
    if (SCALE && on) w[j] *= 0.01f * vox_size_inv[nc / C];
  }
#pragma unroll
  for (int j = 0; j < kTvSlots; ++j) v[j] = at[j] >= 0 ? grid[at[j]] : 0.f;
#pragma unroll
  for (int j = 0; j < kTvSlots; ++j) {
    const float v1 = __shfl_xor_sync(0xffffffffu, v[j], 1);
    const float v2 = __shfl_xor_sync(0xffffffffu, v[j], 2);
    const float v4 = __shfl_xor_sync(0xffffffffu, v[j], 4);
    if (at[j] < 0) continue;
    const int s = ((v[j] > v1) * 2 - 1) + ((v[j] > v2) * 2 - 1) + ((v[j] > v4) * 2 - 1);
    atomicAdd(grad + at[j], w[j] * (float)s);
  }
}

void launch_total_variation_bw(const float* grid, const int64_t* vox_key, float weight, const float* vox_size_inv,
                               bool no_tv_s, uint8_t* active, int64_t N, int C, float* grad, cudaStream_t stream) {
  const int64_t n_slots = 8 * N * (int64_t)C;
  if (n_slots <= 0) return;
  const unsigned g = (unsigned)((n_slots + kTvThreads * kTvSlots - 1) / (kTvThreads * kTvSlots));
  auto run = [&](auto cc) {
    constexpr int CC = decltype(cc)::value;
    if (active) tv_active_kernel<CC><<<g, kTvThreads, 0, stream>>>(n_slots, C, vox_key, grad, active);
    if (no_tv_s)
      tv_grad_kernel<false, CC><<<g, kTvThreads, 0, stream>>>(n_slots, C, grid, vox_key, weight, vox_size_inv,
                                                               active, grad);
    else
      tv_grad_kernel<true, CC><<<g, kTvThreads, 0, stream>>>(n_slots, C, grid, vox_key, weight, vox_size_inv,
                                                              active, grad);
  };
  if (C == 1) run(std::integral_constant<int, 1>());
  else if (C == 3) run(std::integral_constant<int, 3>());
  else run(std::integral_constant<int, 0>());
}

}  // namespace svr
