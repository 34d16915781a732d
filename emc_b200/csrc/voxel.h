// Voxel arithmetic shared by host code and CUDA kernels.
//
// Voxel choice is a discrete decision, so every operation is written with an
// explicit rounding step (device: __fmul_rn/__fadd_rn/__fmaf_rn, which the
// compiler never contracts; host: plain float ops compiled with
// -ffp-contract=off and std::fmaf).  Host and device therefore pick the same
// voxel for the same inputs.
//   rotation matrix   coefficients of emc_cuda.cu:65-85
//   position          u = side/2 + 0.5 + R.c  (emc_cuda.cu:86-88); voxel k is centred at u == k
//   nearest           roundf(u), bounds lower <= k < side: lower = 1 for slicing
//                     (emc_cuda.cu:89-91), 0 for insertion (emc_atomic.cu:56-58)
//   trilinear         corners floor(u) and floor(u)+1, each kept if 0 <= k < side
#pragma once
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define EMC_HD __host__ __device__ __forceinline__
#else
#define EMC_HD inline
#endif

namespace emc_voxel {

EMC_HD float mul(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
EMC_HD float add(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
EMC_HD float sub(float a, float b) {
#ifdef __CUDA_ARCH__
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
EMC_HD float fma(float a, float b, float c) {
#ifdef __CUDA_ARCH__
  return __fmaf_rn(a, b, c);
#else
  return std::fmaf(a, b, c);
#endif
}

EMC_HD void rotation_matrix(const float* q, float* m) {
  const float q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
  const float a = mul(q0, q0), b = mul(q1, q1), c = mul(q2, q2), d = mul(q3, q3);
  const float t12 = mul(mul(2.0f, q1), q2), t03 = mul(mul(2.0f, q0), q3);
  const float t13 = mul(mul(2.0f, q1), q3), t02 = mul(mul(2.0f, q0), q2);
  const float t23 = mul(mul(2.0f, q2), q3), t01 = mul(mul(2.0f, q0), q1);
  m[0] = sub(sub(add(a, b), c), d);
  m[1] = sub(t12, t03);
  m[2] = add(t13, t02);
  m[3] = add(t12, t03);
  m[4] = sub(add(sub(a, b), c), d);
  m[5] = sub(t23, t01);
  m[6] = sub(t13, t02);
  m[7] = add(t23, t01);
  m[8] = add(sub(sub(a, b), c), d);
}

EMC_HD void position(const float* m, int side, float x, float y, float z, float* u) {
  const float c = (float)side / 2.0f + 0.5f;
  u[0] = add(c, fma(m[0], x, fma(m[1], y, mul(m[2], z))));
  u[1] = add(c, fma(m[3], x, fma(m[4], y, mul(m[5], z))));
  u[2] = add(c, fma(m[6], x, fma(m[7], y, mul(m[8], z))));
}

EMC_HD bool nearest(const float* u, int side, int lower, int64_t* v) {
  const int kx = (int)roundf(u[0]), ky = (int)roundf(u[1]), kz = (int)roundf(u[2]);
  if (kx < lower || kx >= side || ky < lower || ky >= side || kz < lower || kz >= side)
    return false;
  *v = ((int64_t)kz * side + ky) * side + kx;
  return true;
}

// Corner c (0..7, bit 0 = x, 1 = y, 2 = z) of the trilinear stencil: its voxel
// and weight, false when it lies outside the grid.  Callers unroll over c, so
// no stencil array is kept.
EMC_HD bool trilinear_corner(const float* u, int side, int c, int64_t* v, float* w) {
  const float fx = floorf(u[0]), fy = floorf(u[1]), fz = floorf(u[2]);
  const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
  const int kx = (int)fx + bx, ky = (int)fy + by, kz = (int)fz + bz;
  if (kx < 0 || kx >= side || ky < 0 || ky >= side || kz < 0 || kz >= side) return false;
  const float ax = u[0] - fx, ay = u[1] - fy, az = u[2] - fz;
  *w = (bx ? ax : 1.0f - ax) * (by ? ay : 1.0f - ay) * (bz ? az : 1.0f - az);
  *v = ((int64_t)kz * side + ky) * side + kx;
  return true;
}

// Returns the number of in-grid corners written to v/w (at most 8).
EMC_HD int trilinear(const float* u, int side, int64_t* v, float* w) {
  const float fx = floorf(u[0]), fy = floorf(u[1]), fz = floorf(u[2]);
  const int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
  const float ax = u[0] - fx, ay = u[1] - fy, az = u[2] - fz;
  int n = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
    const int kx = x0 + bx, ky = y0 + by, kz = z0 + bz;
    if (kx < 0 || kx >= side || ky < 0 || ky >= side || kz < 0 || kz >= side) continue;
    const float wc = (bx ? ax : 1.0f - ax) * (by ? ay : 1.0f - ay) * (bz ? az : 1.0f - az);
    if (wc == 0.0f) continue;
    v[n] = ((int64_t)kz * side + ky) * side + kx;
    w[n] = wc;
    ++n;
  }
  return n;
}

}  // namespace emc_voxel
