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
#include "svr_common.cuh"
#include "svr_kernels.h"

namespace svr {

__global__ void __launch_bounds__(256)
tv_active_kernel(int64_t NC, int C, const int64_t* __restrict__ vox_key, const float* __restrict__ grad,
                 uint8_t* __restrict__ active) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= NC) return;
  const int64_t n = idx / C, c = idx % C;
  bool any = false;
#pragma unroll
  for (int i = 0; i < 8; ++i) any |= grad[vox_key[8 * n + i] * C + c] != 0.f;
  active[idx] = any;
}

template <bool SCALE>
__global__ void __launch_bounds__(256)
tv_grad_kernel(int64_t NC, int C, const float* __restrict__ grid, const int64_t* __restrict__ vox_key, float weight,
               const float* __restrict__ vox_size_inv, const uint8_t* __restrict__ active, float* __restrict__ grad) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= NC) return;
  if (active && !active[idx]) return;
  const int64_t n = idx / C, c = idx % C;
  int64_t key[8];
  float v[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    key[i] = vox_key[8 * n + i];
    v[i] = grid[key[i] * C + c];
  }
  float w = weight;
  if (SCALE) w *= 0.01f * vox_size_inv[n];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int s = ((v[i] > v[i ^ 1]) * 2 - 1) + ((v[i] > v[i ^ 2]) * 2 - 1) + ((v[i] > v[i ^ 4]) * 2 - 1);
    atomicAdd(grad + key[i] * C + c, w * (float)s);
  }
}

void launch_total_variation_bw(const float* grid, const int64_t* vox_key, float weight, const float* vox_size_inv,
                               bool no_tv_s, uint8_t* active, int64_t N, int C, float* grad, cudaStream_t stream) {
  const int64_t NC = N * (int64_t)C;
  if (NC <= 0) return;
  const unsigned g = (unsigned)((NC + 255) / 256);
  if (active) tv_active_kernel<<<g, 256, 0, stream>>>(NC, C, vox_key, grad, active);
  if (no_tv_s) tv_grad_kernel<false><<<g, 256, 0, stream>>>(NC, C, grid, vox_key, weight, vox_size_inv, active, grad);
  else tv_grad_kernel<true><<<g, 256, 0, stream>>>(NC, C, grid, vox_key, weight, vox_size_inv, active, grad);
}

}  // namespace svr
