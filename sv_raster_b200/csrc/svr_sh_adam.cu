// Spherical-harmonics colour, Adam updates and grid-point gathers.
//
// SH: follows computeColorFromSH / _bw (backends/cuda/src/sh_compute.cu:54-176)
// expression for expression, so colours are bit-identical.  Degree is a
// template parameter; fp32 and bf16 coefficient storage are supported.
//
// Adam: unbiased_adam_step_cuda_kernel / biased_... (adam_step.cu:28-102)
// with the host-side double bias correction (adam_step.cu:117-122), plus a
// fused multi-group form that updates several parameter groups in one launch.
//
// Gather: gather_triinterp_geo_params(_bw) / feat (geo_params_gather.cu:22-130).
#include <cuda_bf16.h>

#include "svr_common.cuh"
#include "svr_kernels.h"
#include "svr_sh.cuh"

namespace svr {

template <int DEG, typename TS>
__global__ void __launch_bounds__(256)
sh_eval_kernel(int n_idx, int P, int M, const int64_t* __restrict__ idx, const float* __restrict__ centers,
               const float* __restrict__ cam_pos, const TS* __restrict__ sh0, const TS* __restrict__ shs,
               float* __restrict__ rgbs) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if ((n_idx == 0 && tid >= P) || (n_idx != 0 && tid >= n_idx)) return;
  const int64_t i = (n_idx != 0) ? idx[tid] : tid;
  float dx = centers[3 * i + 0] - cam_pos[0];
  float dy = centers[3 * i + 1] - cam_pos[1];
  float dz = centers[3 * i + 2] - cam_pos[2];
  const float rn = rnorm3df(dx, dy, dz);
  dx = dx * rn; dy = dy * rn; dz = dz * rn;
  const TS* sh = shs + (size_t)i * (M - 1) * 3;
#pragma unroll
  for (int c = 0; c < 3; ++c) rgbs[3 * i + c] = sh_channel<DEG>(dx, dy, dz, ldf(sh0, 3 * i + c), sh, c);
}

template <int DEG>
__global__ void __launch_bounds__(256)
sh_eval_bw_kernel(int n_idx, int P, int M, const int64_t* __restrict__ idx, const float* __restrict__ centers,
                  const float* __restrict__ cam_pos, const float* __restrict__ dL_drgbs, float* __restrict__ dL_dsh0,
                  float* __restrict__ dL_dshs) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if ((n_idx == 0 && tid >= P) || (n_idx != 0 && tid >= n_idx)) return;
  const int64_t i = (n_idx != 0) ? idx[tid] : tid;
  float x = centers[3 * i + 0] - cam_pos[0];
  float y = centers[3 * i + 1] - cam_pos[1];
  float z = centers[3 * i + 2] - cam_pos[2];
  const float rn = rnorm3df(x, y, z);
  x = x * rn; y = y * rn; z = z * rn;
  const float g[3] = {dL_drgbs[3 * i + 0], dL_drgbs[3 * i + 1], dL_drgbs[3 * i + 2]};
  float* d = dL_dshs + (size_t)i * (M - 1) * 3;
  float basis[15];
  const int nb = sh_basis_rest<DEG>(x, y, z, basis);
#pragma unroll
  for (int c = 0; c < 3; ++c) dL_dsh0[3 * i + c] = kC0 * g[c];
#pragma unroll
  for (int k = 0; k < 15; ++k) {
    if (k >= nb) break;
#pragma unroll
    for (int c = 0; c < 3; ++c) d[3 * k + c] = basis[k] * g[c];
  }
}

void launch_sh_eval(int deg, int n_idx, int P, int M, const int64_t* idx, const float* centers, const float* cam_pos,
                    const void* sh0, const void* shs, bool bf16, float* rgbs, cudaStream_t stream) {
  const int n = n_idx != 0 ? n_idx : P;
  if (n <= 0) return;
  const int g = (n + 255) / 256;
#define SVR_SH_L(D)                                                                                            \
  if (bf16)                                                                                                    \
    sh_eval_kernel<D, __nv_bfloat16><<<g, 256, 0, stream>>>(n_idx, P, M, idx, centers, cam_pos,                \
                                                            (const __nv_bfloat16*)sh0, (const __nv_bfloat16*)shs, rgbs); \
  else                                                                                                         \
    sh_eval_kernel<D, float><<<g, 256, 0, stream>>>(n_idx, P, M, idx, centers, cam_pos, (const float*)sh0,     \
                                                    (const float*)shs, rgbs);
  switch (deg) {
    case 0: SVR_SH_L(0) break;
    case 1: SVR_SH_L(1) break;
    case 2: SVR_SH_L(2) break;
    default: SVR_SH_L(3) break;
  }
#undef SVR_SH_L
}

void launch_sh_eval_bw(int deg, int n_idx, int P, int M, const int64_t* idx, const float* centers,
                       const float* cam_pos, const float* dL_drgbs, float* dL_dsh0, float* dL_dshs,
                       cudaStream_t stream) {
  const int n = n_idx != 0 ? n_idx : P;
  if (n <= 0) return;
  const int g = (n + 255) / 256;
  switch (deg) {
    case 0: sh_eval_bw_kernel<0><<<g, 256, 0, stream>>>(n_idx, P, M, idx, centers, cam_pos, dL_drgbs, dL_dsh0, dL_dshs); break;
    case 1: sh_eval_bw_kernel<1><<<g, 256, 0, stream>>>(n_idx, P, M, idx, centers, cam_pos, dL_drgbs, dL_dsh0, dL_dshs); break;
    case 2: sh_eval_bw_kernel<2><<<g, 256, 0, stream>>>(n_idx, P, M, idx, centers, cam_pos, dL_drgbs, dL_dsh0, dL_dshs); break;
    default: sh_eval_bw_kernel<3><<<g, 256, 0, stream>>>(n_idx, P, M, idx, centers, cam_pos, dL_drgbs, dL_dsh0, dL_dshs); break;
  }
}

// ---------------------------------------------------------------------------
// Adam
// ---------------------------------------------------------------------------
__device__ __forceinline__ float adam_lerp(float v0, float v1, float t) {
  return fmaf(t, v1, fmaf(-t, v0, v0));  // (1-t)*v0 + t*v1, adam_step.cu:21-25
}

template <bool SPARSE>
__global__ void __launch_bounds__(256)
adam_unbiased_kernel(int64_t numel, float* __restrict__ param, const float* __restrict__ grad,
                     float* __restrict__ exp_avg, float* __restrict__ exp_avg_sq, float step_size, float beta1,
                     float beta2, float rsqrt_bc2, float eps) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numel) return;
  const float g = grad[i];
  if (SPARSE && g == 0.0f) return;
  float m = exp_avg[i];
  float v = exp_avg_sq[i];
  m = adam_lerp(g, m, beta1);
  v = adam_lerp(g * g, v, beta2);
  const float denom = fmaf(sqrtf(v), rsqrt_bc2, eps);
  const float step = step_size * (m / denom);
  param[i] -= step;
  exp_avg[i] = m;
  exp_avg_sq[i] = v;
}

template <bool SPARSE>
__global__ void __launch_bounds__(256)
adam_biased_kernel(int64_t numel, float* __restrict__ param, const float* __restrict__ grad,
                   float* __restrict__ exp_avg, float* __restrict__ exp_avg_sq, float lr, float beta1, float beta2,
                   float eps) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numel) return;
  const float g = grad[i];
  if (SPARSE && g == 0.0f) return;
  float m = exp_avg[i];
  float v = exp_avg_sq[i];
  m = adam_lerp(g, m, beta1);
  v = adam_lerp(g * g, v, beta2);
  const float denom = sqrtf(v) + eps;
  const float step = lr * (m / denom);
  param[i] -= step;
  exp_avg[i] = m;
  exp_avg_sq[i] = v;
}

void launch_adam(bool biased, bool sparse, int64_t numel, float* param, const float* grad, float* m, float* v,
                 float step_or_lr, float beta1, float beta2, float rsqrt_bc2, float eps, cudaStream_t stream) {
  if (numel <= 0) return;
  const unsigned g = (unsigned)((numel + 255) / 256);
  if (biased) {
    if (sparse) adam_biased_kernel<true><<<g, 256, 0, stream>>>(numel, param, grad, m, v, step_or_lr, beta1, beta2, eps);
    else adam_biased_kernel<false><<<g, 256, 0, stream>>>(numel, param, grad, m, v, step_or_lr, beta1, beta2, eps);
  } else {
    if (sparse)
      adam_unbiased_kernel<true><<<g, 256, 0, stream>>>(numel, param, grad, m, v, step_or_lr, beta1, beta2, rsqrt_bc2, eps);
    else
      adam_unbiased_kernel<false><<<g, 256, 0, stream>>>(numel, param, grad, m, v, step_or_lr, beta1, beta2, rsqrt_bc2, eps);
  }
}

// Fused multi-group Adam: one launch walks every group's elements with
// 4-wide vector access.  Parameters may be fp32 or bf16 (fp32 moments and
// gradients); the per-element arithmetic is the unbiased kernel's.
__global__ void __launch_bounds__(256)
adam_fused_kernel(const __grid_constant__ AdamGroupTable t) {
  const int grp = blockIdx.y;
  if (grp >= t.n) return;
  const AdamGroup& G = t.g[grp];
  // Bias correction: from the host (step_size, rsqrt_bc2) or, for a step
  // counter kept on the device (graph replays), computed here in double
  // exactly as the host would (adam_step.cu:117-122).
  __shared__ float s_step_size, s_rbc2;
  float step_size = G.step_size, rbc2 = G.rsqrt_bc2;
  if (t.d_step) {
    if (threadIdx.x == 0) {
      const double st = (double)*t.d_step;
      s_step_size = (float)(G.lr / (1.0 - pow(t.beta1d, st)));
      s_rbc2 = (float)(1.0 / sqrt(1.0 - pow(t.beta2d, st)));
    }
    __syncthreads();
    step_size = s_step_size;
    rbc2 = s_rbc2;
  }
  const int64_t n4 = G.numel / 4;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < (G.numel + 3) / 4; q += stride) {
    const bool full = q < n4;
    float g4[4], m4[4], v4[4], p4[4];
    if (full) {
      *reinterpret_cast<float4*>(g4) = reinterpret_cast<const float4*>(G.grad)[q];
      *reinterpret_cast<float4*>(m4) = reinterpret_cast<const float4*>(G.exp_avg)[q];
      *reinterpret_cast<float4*>(v4) = reinterpret_cast<const float4*>(G.exp_avg_sq)[q];
      if (G.param_bf16) {
        const uint2 raw = reinterpret_cast<const uint2*>(G.param)[q];
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&raw);
        const float2 a = __bfloat1622float2(h[0]), b = __bfloat1622float2(h[1]);
        p4[0] = a.x; p4[1] = a.y; p4[2] = b.x; p4[3] = b.y;
      } else {
        *reinterpret_cast<float4*>(p4) = reinterpret_cast<const float4*>(G.param)[q];
      }
    } else {
      for (int k = 0; k < 4; ++k) {
        const int64_t i = 4 * q + k;
        const bool ok = i < G.numel;
        g4[k] = ok ? G.grad[i] : 0.f;
        m4[k] = ok ? G.exp_avg[i] : 0.f;
        v4[k] = ok ? G.exp_avg_sq[i] : 0.f;
        p4[k] = ok ? (G.param_bf16 ? __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(G.param)[i])
                                   : reinterpret_cast<const float*>(G.param)[i])
                   : 0.f;
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float g = g4[k];
      if (t.sparse && g == 0.0f) continue;
      float m = adam_lerp(g, m4[k], G.beta1);
      float v = adam_lerp(g * g, v4[k], G.beta2);
      const float denom = fmaf(sqrtf(v), rbc2, G.eps);
      const float step = step_size * (m / denom);
      p4[k] -= step;
      m4[k] = m;
      v4[k] = v;
    }
    if (full) {
      reinterpret_cast<float4*>(G.exp_avg)[q] = *reinterpret_cast<float4*>(m4);
      reinterpret_cast<float4*>(G.exp_avg_sq)[q] = *reinterpret_cast<float4*>(v4);
      if (G.param_bf16) {
        __nv_bfloat162 h[2] = {__floats2bfloat162_rn(p4[0], p4[1]), __floats2bfloat162_rn(p4[2], p4[3])};
        reinterpret_cast<uint2*>(G.param)[q] = *reinterpret_cast<uint2*>(h);
      } else {
        reinterpret_cast<float4*>(G.param)[q] = *reinterpret_cast<float4*>(p4);
      }
    } else {
      for (int k = 0; k < 4; ++k) {
        const int64_t i = 4 * q + k;
        if (i >= G.numel) break;
        G.exp_avg[i] = m4[k];
        G.exp_avg_sq[i] = v4[k];
        if (G.param_bf16) reinterpret_cast<__nv_bfloat16*>(G.param)[i] = __float2bfloat16_rn(p4[k]);
        else reinterpret_cast<float*>(G.param)[i] = p4[k];
      }
    }
  }
}

__global__ void step_increment_kernel(int* d_step) { *d_step += 1; }

void launch_step_increment(int* d_step, cudaStream_t stream) { step_increment_kernel<<<1, 1, 0, stream>>>(d_step); }

void launch_adam_fused(const AdamGroupTable& t, int num_sms, cudaStream_t stream) {
  if (t.n <= 0) return;
  int64_t maxq = 0;
  for (int i = 0; i < t.n; ++i) maxq = std::max<int64_t>(maxq, (t.g[i].numel + 3) / 4);
  if (maxq == 0) return;
  const int64_t want = (maxq + 255) / 256;
  const int cap = std::max(1, num_sms * 8);
  dim3 grid((unsigned)std::min<int64_t>(want, cap), t.n);
  adam_fused_kernel<<<grid, 256, 0, stream>>>(t);
}

// ---------------------------------------------------------------------------
// Grid-point gathers
// ---------------------------------------------------------------------------
// One slot per (cared voxel, corner): the 8 slots of a voxel read its 8 keys
// and write its 8 outputs as one contiguous run, so key reads and output
// stores are coalesced across the warp; only the grid-point reads (and the
// backward's adds) are scattered.  Each thread carries U slots, 256 apart,
// through every load stage together so U scattered reads are in flight.
constexpr int kGatherThreads = 256;

template <int DIM, int U>
__global__ void __launch_bounds__(kGatherThreads)
gather_kernel(int64_t n_slots, const int64_t* __restrict__ vox_key, const int64_t* __restrict__ care_idx,
              const float* __restrict__ grid_pts, float* __restrict__ out) {
  const int64_t base = (int64_t)blockIdx.x * (kGatherThreads * U) + threadIdx.x;
  int64_t slot[U], k[U];
  float v[U][DIM];
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const int64_t t = base + j * kGatherThreads;
    slot[j] = t < n_slots ? 8 * care_idx[t >> 3] + (t & 7) : -1;
  }
#pragma unroll
  for (int j = 0; j < U; ++j) k[j] = slot[j] >= 0 ? vox_key[slot[j]] : 0;
#pragma unroll
  for (int j = 0; j < U; ++j)
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[j][d] = slot[j] >= 0 ? grid_pts[k[j] * DIM + d] : 0.f;
#pragma unroll
  for (int j = 0; j < U; ++j)
    if (slot[j] >= 0)
#pragma unroll
      for (int d = 0; d < DIM; ++d) out[slot[j] * DIM + d] = v[j][d];
}

template <int DIM, int U>
__global__ void __launch_bounds__(kGatherThreads)
gather_bw_kernel(int64_t n_slots, const int64_t* __restrict__ vox_key, const int64_t* __restrict__ care_idx,
                 const float* __restrict__ dL_dvox, float* __restrict__ dL_dgrid) {
  const int64_t base = (int64_t)blockIdx.x * (kGatherThreads * U) + threadIdx.x;
  int64_t slot[U], k[U];
  float g[U][DIM];
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const int64_t t = base + j * kGatherThreads;
    slot[j] = t < n_slots ? 8 * care_idx[t >> 3] + (t & 7) : -1;
  }
#pragma unroll
  for (int j = 0; j < U; ++j) {
    k[j] = slot[j] >= 0 ? vox_key[slot[j]] : 0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) g[j][d] = slot[j] >= 0 ? dL_dvox[slot[j] * DIM + d] : 0.f;
  }
#pragma unroll
  for (int j = 0; j < U; ++j)
    if (slot[j] >= 0)
#pragma unroll
      for (int d = 0; d < DIM; ++d) atomicAdd(dL_dgrid + k[j] * DIM + d, g[j][d]);
}

template <int DIM, int U, class KERNEL>
static void launch_slots(KERNEL kernel, int n_care, const int64_t* vox_key, const int64_t* care_idx, const float* in,
                         float* out, cudaStream_t stream) {
  const int64_t n_slots = 8 * (int64_t)n_care;
  const unsigned g = (unsigned)((n_slots + kGatherThreads * U - 1) / (kGatherThreads * U));
  kernel<<<g, kGatherThreads, 0, stream>>>(n_slots, vox_key, care_idx, in, out);
}

void launch_gather(int dim, int n_care, const int64_t* vox_key, const int64_t* care_idx, const float* grid_pts,
                   float* out, cudaStream_t stream) {
  if (n_care <= 0) return;
  if (dim == 1) launch_slots<1, 4>(gather_kernel<1, 4>, n_care, vox_key, care_idx, grid_pts, out, stream);
  else launch_slots<3, 2>(gather_kernel<3, 2>, n_care, vox_key, care_idx, grid_pts, out, stream);
}

void launch_gather_bw(int dim, int n_care, const int64_t* vox_key, const int64_t* care_idx, const float* dL_dvox,
                      float* dL_dgrid, cudaStream_t stream) {
  if (n_care <= 0) return;
  if (dim == 1) launch_slots<1, 4>(gather_bw_kernel<1, 4>, n_care, vox_key, care_idx, dL_dvox, dL_dgrid, stream);
  else launch_slots<3, 2>(gather_bw_kernel<3, 2>, n_care, vox_key, care_idx, dL_dvox, dL_dgrid, stream);
}

// Batched training over grid points: every voxel's 8 corner densities
// gathered from the grid (fp32 or bf16 grid, fp32 or bf16 output rows), and
// the density gradients [P,8] added back into the grid gradient.  One slot
// per (voxel, corner), U slots per thread, as above; no care list (all
// voxels are rendered by the batched step).
__device__ __forceinline__ float to_f32(float x) { return x; }
__device__ __forceinline__ float to_f32(__nv_bfloat16 x) { return __bfloat162float(x); }
template <class T>
__device__ __forceinline__ T from_f32(float x);
template <>
__device__ __forceinline__ float from_f32<float>(float x) { return x; }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }

template <int U, class GT, class OT>
__global__ void __launch_bounds__(kGatherThreads)
gather_all_geo_kernel(int64_t n_slots, const int64_t* __restrict__ vox_key, const GT* __restrict__ grid_pts,
                      OT* __restrict__ out) {
  const int64_t base = (int64_t)blockIdx.x * (kGatherThreads * U) + threadIdx.x;
  int64_t k[U];
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const int64_t t = base + j * kGatherThreads;
    k[j] = t < n_slots ? vox_key[t] : -1;
  }
  float v[U];
#pragma unroll
  for (int j = 0; j < U; ++j) v[j] = k[j] >= 0 ? to_f32(grid_pts[k[j]]) : 0.f;
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const int64_t t = base + j * kGatherThreads;
    if (t < n_slots) out[t] = from_f32<OT>(v[j]);
  }
}

template <int U>
__global__ void __launch_bounds__(kGatherThreads)
scatter_all_geo_kernel(int64_t n_slots, const int64_t* __restrict__ vox_key, const float* __restrict__ dL_dgeos,
                       float* __restrict__ dL_dgrid) {
  const int64_t base = (int64_t)blockIdx.x * (kGatherThreads * U) + threadIdx.x;
  int64_t k[U];
  float g[U];
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const int64_t t = base + j * kGatherThreads;
    k[j] = t < n_slots ? vox_key[t] : -1;
    g[j] = t < n_slots ? dL_dgeos[t] : 0.f;
  }
#pragma unroll
  for (int j = 0; j < U; ++j)
    if (k[j] >= 0 && g[j] != 0.f) atomicAdd(dL_dgrid + k[j], g[j]);
}

void launch_gather_all_geo(int64_t P, const int64_t* vox_key, const void* grid_pts, bool grid_bf16, void* out,
                           bool out_bf16, cudaStream_t stream) {
  if (P <= 0) return;
  constexpr int U = 4;
  const int64_t n_slots = 8 * P;
  const unsigned g = (unsigned)((n_slots + kGatherThreads * U - 1) / (kGatherThreads * U));
  using bf = __nv_bfloat16;
  if (grid_bf16 && out_bf16)
    gather_all_geo_kernel<U, bf, bf><<<g, kGatherThreads, 0, stream>>>(n_slots, vox_key, (const bf*)grid_pts, (bf*)out);
  else if (grid_bf16)
    gather_all_geo_kernel<U, bf, float><<<g, kGatherThreads, 0, stream>>>(n_slots, vox_key, (const bf*)grid_pts,
                                                                          (float*)out);
  else if (out_bf16)
    gather_all_geo_kernel<U, float, bf><<<g, kGatherThreads, 0, stream>>>(n_slots, vox_key, (const float*)grid_pts,
                                                                          (bf*)out);
  else
    gather_all_geo_kernel<U, float, float><<<g, kGatherThreads, 0, stream>>>(n_slots, vox_key,
                                                                             (const float*)grid_pts, (float*)out);
}

void launch_scatter_all_geo(int64_t P, const int64_t* vox_key, const float* dL_dgeos, float* dL_dgrid,
                            cudaStream_t stream) {
  if (P <= 0) return;
  constexpr int U = 4;
  const int64_t n_slots = 8 * P;
  const unsigned g = (unsigned)((n_slots + kGatherThreads * U - 1) / (kGatherThreads * U));
  scatter_all_geo_kernel<U><<<g, kGatherThreads, 0, stream>>>(n_slots, vox_key, dL_dgeos, dL_dgrid);
}

}  // namespace svr
