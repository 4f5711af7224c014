// Voxel projection: near-sphere cull, 8-corner projection to a packed pixel
// bbox, camera-quadrant bitset and duplicate count.
//
// Follows preprocessCUDA (backends/cuda/src/preprocess.cu:24-132) with the
// same arithmetic (svr_project.cuh), but one launch covers many views
// (gridDim.y) and camera matrices are staged once per CTA in shared memory.
#include "svr_common.cuh"
#include "svr_views.cuh"
#include "svr_kernels.h"
#include "svr_project.cuh"

namespace svr {

__global__ void __launch_bounds__(256)
preprocess_kernel(const __grid_constant__ ViewTable views, int P,
                  const float* __restrict__ centers, const float* __restrict__ lengths,
                  int32_t* __restrict__ out_ndup,       // [V*P] or nullptr
                  uint32_t* __restrict__ ndup,          // [V*P]
                  uint2* __restrict__ bboxes,           // [V*P]
                  uint32_t* __restrict__ quads)         // [V*P]
{
  const int view = blockIdx.y;
  const ViewParams& vp = views.v[view];
  __shared__ float s_m[24];
  if (threadIdx.x < 12) s_m[threadIdx.x] = vp.w2c[threadIdx.x];
  else if (threadIdx.x < 24) s_m[threadIdx.x] = vp.c2w[threadIdx.x - 12];
  __syncthreads();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= P) return;
  const size_t o = (size_t)view * P + idx;
  const Projection pr = project_voxel(vp, s_m, s_m + 12, centers[3 * (size_t)idx + 0], centers[3 * (size_t)idx + 1],
                                      centers[3 * (size_t)idx + 2], lengths[idx]);
  if (out_ndup) out_ndup[o] = (int32_t)pr.n;
  ndup[o] = pr.n;
  bboxes[o] = pr.bbox;
  quads[o] = pr.quads;
}

void launch_preprocess(const ViewTable& views, int P, const float* centers, const float* lengths,
                       int32_t* out_ndup, uint32_t* ndup, uint2* bboxes, uint32_t* quads,
                       cudaStream_t stream) {
  if (P <= 0 || views.n <= 0) return;
  dim3 grid((P + 255) / 256, views.n);
  preprocess_kernel<<<grid, 256, 0, stream>>>(views, P, centers, lengths, out_ndup, ndup, bboxes, quads);
}

}  // namespace svr
