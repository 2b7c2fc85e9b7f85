// SH basis, its gradient, quaternion to matrix and SH storage loads, shared by
// the preprocess and chain-rule kernels. Formulas: shaders/train_types.glsl
// (sh_basis :97-123, sh_basis_gradient :126-153, train_quat_to_mat :172-177).
// Products are evaluated left to right, one rounding each, as written there.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "kernels.cuh"

namespace sb {

__device__ __forceinline__ void sh_basis(float x, float y, float z, int degree, float b[16]) {
  const float C1 = 0.4886025119029199f;
  const float xx = x * x, yy = y * y, zz = z * z;
  b[0] = 0.28209479177387814f;
  if (degree > 0) {
    b[1] = -C1 * y;
    b[2] = C1 * z;
    b[3] = -C1 * x;
  }
  if (degree > 1) {
    b[4] = 1.0925484305920792f * x * y;
    b[5] = -1.0925484305920792f * y * z;
    b[6] = 0.31539156525252005f * (2.0f * zz - xx - yy);
    b[7] = -1.0925484305920792f * x * z;
    b[8] = 0.5462742152960396f * (xx - yy);
  }
  if (degree > 2) {
    b[9] = -0.5900435899266435f * y * (3.0f * xx - yy);
    b[10] = 2.890611442640554f * x * y * z;
    b[11] = -0.4570457994644658f * y * (4.0f * zz - xx - yy);
    b[12] = 0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    b[13] = -0.4570457994644658f * x * (4.0f * zz - xx - yy);
    b[14] = 1.445305721320277f * z * (xx - yy);
    b[15] = -0.5900435899266435f * x * (xx - 3.0f * yy);
  }
}

// d(basis_k)/d(dir), three components per k.
__device__ __forceinline__ void sh_basis_gradient(float x, float y, float z, int degree, float g[16][3]) {
  const float C1 = 0.4886025119029199f, A = 1.0925484305920792f, K = 0.31539156525252005f, L = 0.5462742152960396f;
  const float C = -0.5900435899266435f, E = 2.890611442640554f, F = -0.4570457994644658f, G = 0.3731763325901154f,
              H = 1.445305721320277f;
  const float xx = x * x, yy = y * y, zz = z * z;
#define SB_SET(k, a, b_, c) \
  g[k][0] = (a);            \
  g[k][1] = (b_);           \
  g[k][2] = (c);
  SB_SET(0, 0.f, 0.f, 0.f)
  if (degree > 0) {
    SB_SET(1, 0.f, -C1, 0.f)
    SB_SET(2, 0.f, 0.f, C1)
    SB_SET(3, -C1, 0.f, 0.f)
  }
  if (degree > 1) {
    SB_SET(4, A * y, A * x, 0.f)
    SB_SET(5, -A * 0.f, -A * z, -A * y)
    SB_SET(6, K * (-2.0f * x), K * (-2.0f * y), K * (4.0f * z))
    SB_SET(7, -A * z, -A * 0.f, -A * x)
    SB_SET(8, L * (2.0f * x), L * (-2.0f * y), 0.f)
  }
  if (degree > 2) {
    SB_SET(9, C * (6.0f * x * y), C * (3.0f * xx - 3.0f * yy), 0.f)
    SB_SET(10, E * (y * z), E * (x * z), E * (x * y))
    SB_SET(11, F * (-2.0f * x * y), F * (4.0f * zz - xx - 3.0f * yy), F * (8.0f * y * z))
    SB_SET(12, G * (-6.0f * x * z), G * (-6.0f * y * z), G * (6.0f * zz - 3.0f * xx - 3.0f * yy))
    SB_SET(13, F * (4.0f * zz - 3.0f * xx - yy), F * (-2.0f * x * y), F * (8.0f * x * z))
    SB_SET(14, H * (2.0f * x * z), H * (-2.0f * y * z), H * (xx - yy))
    SB_SET(15, C * (3.0f * xx - 3.0f * yy), C * (-6.0f * x * y), 0.f)
  }
#undef SB_SET
}

// Rotation matrix of a unit quaternion (w, x, y, z), row-major: m[r][c].
__device__ __forceinline__ void quat_to_matrix(float w, float x, float y, float z, float m[3][3]) {
  const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y, wz = w * z;
  // GLSL mat3 columns (1-2(yy+zz), 2(xy+wz), 2(xz-wy)), ... transposed into rows.
  m[0][0] = 1.0f - 2.0f * (yy + zz);
  m[1][0] = 2.0f * (xy + wz);
  m[2][0] = 2.0f * (xz - wy);
  m[0][1] = 2.0f * (xy - wz);
  m[1][1] = 1.0f - 2.0f * (xx + zz);
  m[2][1] = 2.0f * (yz + wx);
  m[0][2] = 2.0f * (xz + wy);
  m[1][2] = 2.0f * (yz - wx);
  m[2][2] = 1.0f - 2.0f * (xx + yy);
}

template <ShStore S> __device__ __forceinline__ float load_sh_rest(const void *p, size_t idx);
template <> __device__ __forceinline__ float load_sh_rest<ShStore::F32>(const void *p, size_t idx) {
  return static_cast<const float *>(p)[idx];
}
template <> __device__ __forceinline__ float load_sh_rest<ShStore::BF16>(const void *p, size_t idx) {
  const uint32_t bits = static_cast<const uint16_t *>(p)[idx];
  return __uint_as_float(bits << 16);
}
template <> __device__ __forceinline__ float load_sh_rest<ShStore::F16>(const void *p, size_t idx) {
  return __half2float(static_cast<const __half *>(p)[idx]);
}

// Element e (= 3 (k - 1) + c) of Gaussian i's row of higher coefficients.
__host__ __device__ __forceinline__ size_t sh_rest_at(uint32_t i, uint32_t e, uint32_t restStride) {
  return (size_t)i * restStride + e;
}

// Coefficient k (0 = DC), channel c, of Gaussian i.
template <ShStore S> __device__ __forceinline__ float sh_coefficient(const Params &p, uint32_t i, int k, int c) {
  if (k == 0) return p.shDc[(size_t)c * p.planeStride + i];
  return load_sh_rest<S>(p.shRest, sh_rest_at(i, (uint32_t)((k - 1) * 3 + c), p.restStride));
}

} // namespace sb
