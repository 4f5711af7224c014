// Voxel projection: near-sphere cull, 8-corner projection to a packed pixel
// bbox, camera-quadrant bitset and duplicate count.
//
// Follows preprocessCUDA (backends/cuda/src/preprocess.cu:24-132) with the
// same arithmetic, but: one launch covers many views (gridDim.y), camera
// matrices are staged once per CTA in shared memory, and an impossible tile
// count raises nothing (it cannot occur: the bbox test above it guarantees
// min <= max, so the clamped tile rectangle is never empty).
#include "svr_common.cuh"
#include "svr_views.cuh"
#include "svr_kernels.h"

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

  const float vcx = centers[3 * (size_t)idx + 0];
  const float vcy = centers[3 * (size_t)idx + 1];
  const float vcz = centers[3 * (size_t)idx + 2];
  const float vr = 0.5f * lengths[idx];
  const float* w2c = s_m;
  const float rox = s_m[12 + 3], roy = s_m[12 + 7], roz = s_m[12 + 11];

  uint32_t n = 0, qbits = 0;
  uint2 bb = make_uint2(0u, 0u);
  const float near = vp.near_plane;

  // Near-plane "sphere" test on the voxel centre (preprocess.cu:62-65).
  const float rx = vcx - rox, ry = vcy - roy, rz = vcz - roz;
  if (!(rx * rx + ry * ry + rz * rz < near * near)) {
    float umin = 1e9f, vmin = 1e9f, umax = -1e9f, vmax = -1e9f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float sx = (float)(((i & 4) >> 2) * 2 - 1);
      const float sy = (float)(((i & 2) >> 1) * 2 - 1);
      const float sz = (float)(((i & 1)) * 2 - 1);
      const float wx = vcx + vr * sx, wy = vcy + vr * sy, wz = vcz + vr * sz;
      const float camx = w2c[0] * wx + w2c[1] * wy + w2c[2] * wz + w2c[3];
      const float camy = w2c[4] * wx + w2c[5] * wy + w2c[6] * wz + w2c[7];
      const float camz = w2c[8] * wx + w2c[9] * wy + w2c[10] * wz + w2c[11];
      if (camz < near) continue;
      const float inv_z = 1.0f / camz;
      const float u = camx * inv_z, v = camy * inv_z;
      const uint32_t q = ((uint32_t)(wx < rox) << 2) | ((uint32_t)(wy < roy) << 1) | (uint32_t)(wz < roz);
      umin = fminf(umin, u); vmin = fminf(vmin, v);
      umax = fmaxf(umax, u); vmax = fmaxf(vmax, v);
      qbits |= (1u << q);
    }
    const float cxh = vp.cx - 0.5f, cyh = vp.cy - 0.5f;
    const float bx0 = fmaxf(vp.focal_x * umin + cxh, 0.0f);
    const float by0 = fmaxf(vp.focal_y * vmin + cyh, 0.0f);
    const float bx1 = fminf(vp.focal_x * umax + cxh, (float)vp.W);
    const float by1 = fminf(vp.focal_y * vmax + cyh, (float)vp.H);
    if (!(bx0 > bx1 || by0 > by1)) {
      bb.x = (((uint32_t)lrintf(bx0)) << 16) | ((uint32_t)lrintf(by0));
      bb.y = (((uint32_t)lrintf(bx1)) << 16) | ((uint32_t)lrintf(by1));
      int tx0, ty0, tx1, ty1;
      bbox_tile_rect(bb, vp.grid_x, vp.grid_y, tx0, ty0, tx1, ty1);
      const int tiles = (1 + ty1 - ty0) * (1 + tx1 - tx0);
      n = (uint32_t)tiles * (uint32_t)__popc(qbits);
    } else {
      qbits = 0;
    }
  } else {
    qbits = 0;
  }
  if (out_ndup) out_ndup[o] = (int32_t)n;
  ndup[o] = n;
  bboxes[o] = bb;
  quads[o] = qbits;
}

void launch_preprocess(const ViewTable& views, int P, const float* centers, const float* lengths,
                       int32_t* out_ndup, uint32_t* ndup, uint2* bboxes, uint32_t* quads,
                       cudaStream_t stream) {
  if (P <= 0 || views.n <= 0) return;
  dim3 grid((P + 255) / 256, views.n);
  preprocess_kernel<<<grid, 256, 0, stream>>>(views, P, centers, lengths, out_ndup, ndup, bboxes, quads);
}

}  // namespace svr
