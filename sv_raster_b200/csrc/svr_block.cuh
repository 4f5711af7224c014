// CTA- and warp-level helpers shared by the scan, sort and segment-sort kernels.
#pragma once

#include <cstdint>

namespace svr {

// Exclusive scan of one 32-bit value per thread over a CTA of NT threads.
template <int NT, typename T>
__device__ __forceinline__ T block_exclusive_scan(T x, T* s_warp /*[NT/32]*/, T& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = (lane < NT / 32) ? s_warp[lane] : T(0);
    T winc = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, winc, o);
      if (lane >= o) winc += y;
    }
    if (lane < NT / 32) s_warp[lane] = winc - w;  // exclusive warp offsets
    if (lane == NT / 32 - 1) s_warp[NT / 32] = winc;
  }
  __syncthreads();
  T res = s_warp[warp] + inc - x;
  total = s_warp[NT / 32];
  __syncthreads();
  return res;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

}  // namespace svr
