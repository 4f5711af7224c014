// Real spherical-harmonics colour of one voxel, degrees 0-3, and its basis.
// Expression order follows computeColorFromSH (backends/cuda/src/sh_compute.cu:54-106)
// so results are bit-identical to the reference's.
#pragma once

#include <cuda_bf16.h>

namespace svr {

// Real SH basis normalisation constants (degrees 0-3).
__device__ constexpr float kC0 = 0.28209479177387814f;
__device__ constexpr float kC1 = 0.4886025119029199f;
__device__ constexpr float kC2[5] = {1.0925484305920792f, -1.0925484305920792f, 0.31539156525252005f,
                                     -1.0925484305920792f, 0.5462742152960396f};
__device__ constexpr float kC3[7] = {-0.5900435899266435f, 2.890611442640554f, -0.4570457994644658f,
                                     0.3731763325901154f, -0.4570457994644658f, 1.445305721320277f,
                                     -0.5900435899266435f};

template <typename TS>
__device__ __forceinline__ float ldf(const TS* p, size_t i) {
  if constexpr (sizeof(TS) == 2) return __bfloat162float(p[i]);
  else return p[i];
}

// rgb of one channel `c`; `sh` points at the voxel's (M-1) x 3 rest coefficients.
template <int DEG, typename TS>
__device__ __forceinline__ float sh_channel(float x, float y, float z, float base0, const TS* sh, int c) {
  float r = kC0 * base0;
  if (DEG > 0) {
    r = r - kC1 * y * ldf(sh, 0 * 3 + c) + kC1 * z * ldf(sh, 1 * 3 + c) - kC1 * x * ldf(sh, 2 * 3 + c);
    if (DEG > 1) {
      const float xx = x * x, yy = y * y, zz = z * z;
      const float xy = x * y, yz = y * z, xz = x * z;
      r = r + kC2[0] * xy * ldf(sh, 3 * 3 + c) + kC2[1] * yz * ldf(sh, 4 * 3 + c) +
          kC2[2] * (2.0f * zz - xx - yy) * ldf(sh, 5 * 3 + c) + kC2[3] * xz * ldf(sh, 6 * 3 + c) +
          kC2[4] * (xx - yy) * ldf(sh, 7 * 3 + c);
      if (DEG > 2) {
        r = r + kC3[0] * y * (3.0f * xx - yy) * ldf(sh, 8 * 3 + c) + kC3[1] * xy * z * ldf(sh, 9 * 3 + c) +
            kC3[2] * y * (4.0f * zz - xx - yy) * ldf(sh, 10 * 3 + c) +
            kC3[3] * z * (2.0f * zz - 3.0f * xx - 3.0f * yy) * ldf(sh, 11 * 3 + c) +
            kC3[4] * x * (4.0f * zz - xx - yy) * ldf(sh, 12 * 3 + c) + kC3[5] * z * (xx - yy) * ldf(sh, 13 * 3 + c) +
            kC3[6] * x * (xx - 3.0f * yy) * ldf(sh, 14 * 3 + c);
      }
    }
  }
  r = r + 0.5f;
  r *= (r > 0.0f);
  return r;
}

// Basis values b_1..b_15 (the degree-0 term is kC0) at a unit direction:
// the SH backward multiplies these by dL/drgb (sh_compute.cu:110-176).
template <int DEG>
__device__ __forceinline__ int sh_basis_rest(float x, float y, float z, float basis[15]) {
  int nb = 0;
  if (DEG > 0) {
    basis[0] = -kC1 * y;
    basis[1] = kC1 * z;
    basis[2] = -kC1 * x;
    nb = 3;
    if (DEG > 1) {
      const float xx = x * x, yy = y * y, zz = z * z;
      const float xy = x * y, yz = y * z, xz = x * z;
      basis[3] = kC2[0] * xy;
      basis[4] = kC2[1] * yz;
      basis[5] = kC2[2] * (2.f * zz - xx - yy);
      basis[6] = kC2[3] * xz;
      basis[7] = kC2[4] * (xx - yy);
      nb = 8;
      if (DEG > 2) {
        basis[8] = kC3[0] * y * (3.f * xx - yy);
        basis[9] = kC3[1] * xy * z;
        basis[10] = kC3[2] * y * (4.f * zz - xx - yy);
        basis[11] = kC3[3] * z * (2.f * zz - 3.f * xx - 3.f * yy);
        basis[12] = kC3[4] * x * (4.f * zz - xx - yy);
        basis[13] = kC3[5] * z * (xx - yy);
        basis[14] = kC3[6] * x * (xx - 3.f * yy);
        nb = 15;
      }
    }
  }
  return nb;
}

}  // namespace svr
