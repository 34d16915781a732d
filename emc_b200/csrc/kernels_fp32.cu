// FP32 CUDA-core kernels: expand, the likelihood / scaling / slice-average
// contractions as register-tiled FP32 kernels, softmax, insertion and model
// normalisation.  This is the plain-FP32 path of the engine and the engine
// behind the reference-compatible API in legacy.cu.
#include <cfloat>
#include <cstdint>

#include "fixed.cuh"
#include "kernels.cuh"
#include "tile.cuh"
#include "voxel.h"

namespace emc {
namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum of one double per thread over the block (blockDim.x multiple of 32).
__device__ double block_sum(double v, double* red) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; ++i) s += red[i];
  return s;  // valid on thread 0
}

__device__ float block_max(float v, float* red) {
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  float s = -FLT_MAX;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; ++i) s = fmaxf(s, red[i]);
  return s;
}

// ------------------------------------------------------------------ expand --
// One block per rotation; threads stride over pixels.  emc_cuda.cu:51-111 for
// the nearest mode (exclusive lower bound), trilinear otherwise.
// Slice value W at continuous voxel position u (0 outside the grid).
template <int INTERP>
__device__ __forceinline__ float gather(const float* __restrict__ model, const float* u, int side) {
  if (INTERP == 0) {
    int64_t v;
    return emc_voxel::nearest(u, side, 1, &v) ? __ldg(model + v) : 0.0f;
  }
  float acc = 0.0f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    int64_t v;
    float w;
    if (emc_voxel::trilinear_corner(u, side, c, &v, &w) && w != 0.0f)
      acc = fmaf(w, __ldg(model + v), acc);
  }
  return acc;
}

// Trilinear through the stencil table (launch_tri_table): the 8 corner values
// of base voxel floor(u) in one aligned 32-byte load, 0 for corners outside
// the grid.  The same FMAs in the same corner order as gather<1>: a corner
// that gather<1> skips (outside, or weight 0) adds w * 0 or 0 * value here,
// which leaves the sum unchanged, so the result is bit for bit the same.
__device__ __forceinline__ float gather_tri(const float4* __restrict__ tri, const float* u,
                                            int side) {
  const float fx = floorf(u[0]), fy = floorf(u[1]), fz = floorf(u[2]);
  const int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
  if (x0 < -1 || x0 >= side || y0 < -1 || y0 >= side || z0 < -1 || z0 >= side) return 0.0f;
  const int64_t s1 = side + 1;
  const int64_t e = ((int64_t)(z0 + 1) * s1 + (y0 + 1)) * s1 + (x0 + 1);
  const float4 lo = __ldg(tri + 2 * e), hi = __ldg(tri + 2 * e + 1);
  const float val[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
  const float ax = u[0] - fx, ay = u[1] - fy, az = u[2] - fz;
  float acc = 0.0f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
    const float w = (bx ? ax : 1.0f - ax) * (by ? ay : 1.0f - ay) * (bz ? az : 1.0f - az);
    acc = fmaf(w, val[c], acc);
  }
  return acc;
}

// tri[2e], tri[2e + 1] = the model at the 8 corners (bit 0: x + 1, bit 1:
// y + 1, bit 2: z + 1; 0 outside the grid) of base voxel e = (z0 + 1, y0 + 1,
// x0 + 1) over [-1, side)^3.
__global__ void tri_table_kernel(const float* __restrict__ model, int side, float4* tri) {
  const int64_t s1 = side + 1;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= s1 * s1 * s1) return;
  const int x0 = (int)(e % s1) - 1, y0 = (int)((e / s1) % s1) - 1, z0 = (int)(e / (s1 * s1)) - 1;
  float v[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int kx = x0 + (c & 1), ky = y0 + ((c >> 1) & 1), kz = z0 + ((c >> 2) & 1);
    const bool in = kx >= 0 && kx < side && ky >= 0 && ky < side && kz >= 0 && kz < side;
    v[c] = in ? model[((int64_t)kz * side + ky) * side + kx] : 0.0f;
  }
  tri[2 * e] = make_float4(v[0], v[1], v[2], v[3]);
  tri[2 * e + 1] = make_float4(v[4], v[5], v[6], v[7]);
}

// Four pixels per thread and iteration: their gathers are independent, so
// four L2 round trips are in flight per thread.
constexpr int kExpandUnroll = 4;
template <int INTERP, int OUT>
__global__ void __launch_bounds__(kBlock) expand_kernel(const ExpandArgs a) {
  __shared__ double red[32];
  const int64_t r = blockIdx.x;
  float m[9];
  emc_voxel::rotation_matrix(a.quat + 4 * r, m);
  double stat = 0.0;
  const int64_t step = (int64_t)blockDim.x * kExpandUnroll;
  for (int64_t i0 = threadIdx.x; i0 < a.ld; i0 += step) {
    float w[kExpandUnroll];
#pragma unroll
    for (int u = 0; u < kExpandUnroll; ++u) {
      const int64_t i = i0 + (int64_t)u * blockDim.x;
      w[u] = 0.0f;
      if (i < a.npix) {
        float pos[3];
        emc_voxel::position(m, a.side, __ldg(a.cx + i), __ldg(a.cy + i), __ldg(a.cz + i), pos);
        w[u] = (INTERP == 1 && a.tri) ? gather_tri(a.tri, pos, a.side)
                                      : gather<INTERP>(a.model, pos, a.side);
      }
    }
#pragma unroll
    for (int u = 0; u < kExpandUnroll; ++u) {
      const int64_t i = i0 + (int64_t)u * blockDim.x;
      if (i < a.ld) {
        const bool real = i < a.npix;
        if (real && a.stat != STAT_NONE && (!a.stat_mask || a.stat_mask[i] != 0))
          stat += a.stat == STAT_SUMSQ ? (double)w[u] * w[u] : (double)w[u];
        const int64_t o = r * a.ld + i;
        if (OUT == EXP_F32) {
          a.out_f32[o] = w[u];
        } else if (OUT == EXP_LOG_F32) {
          a.out_f32[o] = real ? logf(fmaxf(w[u], a.floor_)) : 0.0f;
        } else {
          const float x = real ? (a.log_split ? logf(fmaxf(w[u], a.floor_)) : w[u]) : 0.0f;
          const __half hi = __float2half_rn(x);
          a.out_hi[o] = hi;
          a.out_lo[o] = __float2half_rn(x - __half2float(hi));
        }
      }
    }
  }
  if (a.rowstat) {
    const double s = block_sum(stat, red);
    if (threadIdx.x == 0) a.rowstat[r] = s;
  }
}

// The operand value of the split expansion and its FP16 hi / lo halves,
// packed hi | lo << 16.
__device__ __forceinline__ uint32_t split_bits(float w, float floor_, int log_split) {
  const float x = log_split ? logf(fmaxf(w, floor_)) : w;
  const __half hi = __float2half_rn(x);
  const __half lo = __float2half_rn(x - __half2float(hi));
  return (uint32_t)__half_as_ushort(hi) | ((uint32_t)__half_as_ushort(lo) << 16);
}

__global__ void expand_table_kernel(const float* model, int64_t M, float floor_, int log_split,
                                    uint2* tab) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v > M) return;
  const float w = v < M ? model[v] : 0.0f;
  tab[v] = make_uint2(__float_as_uint(w), split_bits(w, floor_, log_split));
}

// Nearest-voxel expansion into the FP16 hi + lo operands through the voxel
// table: one 8-byte gather per pixel gives the slice value (for the row
// statistic) and its split operand, so no logarithm or split runs per
// element; each thread takes pixel pairs and writes them as half2.  Outputs
// are those of expand_kernel<0, EXP_F16_SPLIT> bit for bit.
__global__ void __launch_bounds__(kBlock) expand_tab_kernel(const ExpandArgs a) {
  __shared__ double red[32];
  const int64_t r = blockIdx.x;
  float m[9];
  emc_voxel::rotation_matrix(a.quat + 4 * r, m);
  const int64_t M = (int64_t)a.side * a.side * a.side;
  const int npix = (int)a.npix, npairs = (int)(a.ld / 2);
  __half2* hi_row = reinterpret_cast<__half2*>(a.out_hi + r * a.ld);
  __half2* lo_row = reinterpret_cast<__half2*>(a.out_lo + r * a.ld);
  double stat = 0.0;
  for (int p0 = threadIdx.x; p0 < npairs; p0 += 2 * kBlock) {
    uint2 t[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = 2 * (p0 + (u >> 1) * kBlock) + (u & 1);
      t[u] = make_uint2(0u, 0u);  // padding columns: zero
      if (i < npix) {
        float pos[3];
        emc_voxel::position(m, a.side, __ldg(a.cx + i), __ldg(a.cy + i), __ldg(a.cz + i), pos);
        int64_t v;
        if (!emc_voxel::nearest(pos, a.side, 1, &v)) v = M;
        t[u] = __ldg(a.tab + v);
      }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int pp = p0 + h * kBlock;
      if (pp >= npairs) continue;
#pragma unroll
      for (int e = 0; e < 2; ++e)
        if (2 * pp + e < npix && a.stat != STAT_NONE) {
          const float w = __uint_as_float(t[2 * h + e].x);
          stat += a.stat == STAT_SUMSQ ? (double)w * w : (double)w;
        }
      const uint32_t b0 = t[2 * h].y, b1 = t[2 * h + 1].y;
      hi_row[pp] = __halves2half2(__ushort_as_half((unsigned short)(b0 & 0xFFFFu)),
                                  __ushort_as_half((unsigned short)(b1 & 0xFFFFu)));
      lo_row[pp] = __halves2half2(__ushort_as_half((unsigned short)(b0 >> 16)),
                                  __ushort_as_half((unsigned short)(b1 >> 16)));
    }
  }
  if (a.rowstat) {
    const double s = block_sum(stat, red);
    if (threadIdx.x == 0) a.rowstat[r] = s;
  }
}

__device__ __forceinline__ int64_t col_of(const int32_t* pix, int64_t j) { return pix ? pix[j] : j; }

// Likelihood: rows = rotations, columns = patterns, reduction over pixels.
struct OpLL {
  using Acc = double;
  static constexpr bool kBKMajor = true;
  LLArgs p;
  __device__ int64_t ksize() const { return p.npa; }
  __device__ float a(int64_t r, int64_t j) const {
    return (r < p.R && j < p.npa) ? __ldg(p.A + r * p.ldA + col_of(p.pix, j)) : 0.0f;
  }
  __device__ float b(int64_t n, int64_t j) const {
    if (n >= p.N || j >= p.npa) return 0.0f;
    const float k = __ldg(p.K + n * p.ldK + col_of(p.pix, j));
    return p.poisson ? k : k / __ldg(p.scaling + n);  // gaussian: image / scaling (emc_cuda.cu:121)
  }
  // inner(acc, a, b): each likelihood's own term, in OpLLGauss / OpLLPoisson
  __device__ void epilogue(double (&acc)[8][4], int64_t r0, int64_t n0, float*) const {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int64_t r = r0 + i;
      if (r >= p.R) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t n = n0 + j;
        if (n >= p.N) continue;
        const double v = p.poisson ? acc[i][j] - (double)p.scaling[n] * p.rowstat[r]
                                   : -acc[i][j] * p.gauss_inv;
        if (p.LL64)
          p.LL64[r * p.ldLL + n] = v;
        else
          p.LL[r * p.ldLL + n] = (float)v;
      }
    }
  }
};
struct OpLLGauss : OpLL {
  static __device__ __forceinline__ float inner(float acc, float a, float b) {
    const float d = a - b;
    return fmaf(d, d, acc);
  }
};
struct OpLLPoisson : OpLL {
  static __device__ __forceinline__ float inner(float acc, float a, float b) { return fmaf(a, b, acc); }
};

// Gaussian scaling denominator: sum_r P_rp sum_j S_rj K_pj, reduced over the
// tile's rows in the epilogue.
struct OpCross {
  using Acc = float;
  static constexpr bool kBKMajor = true;
  CrossArgs p;
  __device__ int64_t ksize() const { return p.npa; }
  __device__ float a(int64_t r, int64_t j) const {
    return (r < p.R && j < p.npa) ? __ldg(p.S + r * p.ldS + col_of(p.pix, j)) : 0.0f;
  }
  __device__ float b(int64_t n, int64_t j) const {
    return (n < p.N && j < p.npa) ? __ldg(p.K + n * p.ldK + col_of(p.pix, j)) : 0.0f;
  }
  static __device__ __forceinline__ float inner(float acc, float a, float b) { return fmaf(a, b, acc); }
  __device__ void epilogue(float (&acc)[8][4], int64_t r0, int64_t n0, float* smem) const {
    double* red = reinterpret_cast<double*>(smem);  // [16][64]
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t n = n0 + j;
      double s = 0;
      if (n < p.N)
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int64_t r = r0 + i;
          if (r < p.R) s += (double)__ldg(p.P + r * p.N + n) * acc[i][j];
        }
      red[ty * 64 + tx * 4 + j] = s;
    }
    __syncthreads();
    if (threadIdx.x < 64) {
      const int64_t n = (int64_t)blockIdx.x * TN + threadIdx.x;
      double s = 0;
      for (int k = 0; k < 16; ++k) s += red[k * 64 + threadIdx.x];
      if (n < p.N) p.den_part[(int64_t)blockIdx.y * p.N + n] = s;
    }
  }
};

// Slice average: rows = rotations, columns = pixels, reduction over patterns.
struct OpCompress {
  using Acc = float;
  static constexpr bool kBKMajor = false;
  CompressArgs p;
  __device__ int64_t ksize() const { return p.N; }
  __device__ float a(int64_t r, int64_t k) const {
    return (r < p.R && k < p.N) ? __ldg(p.P + r * p.N + k) : 0.0f;
  }
  __device__ float b(int64_t j, int64_t k) const {
    return (j < p.npa && k < p.N) ? __ldg(p.K + k * p.ldK + col_of(p.pix, j)) / __ldg(p.scaling + k)
                                  : 0.0f;
  }
  static __device__ __forceinline__ float inner(float acc, float a, float b) { return fmaf(a, b, acc); }
  __device__ void epilogue(float (&acc)[8][4], int64_t r0, int64_t j0, float*) const {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int64_t r = r0 + i;
      if (r >= p.R) continue;
      const float T = p.T[r];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t jj = j0 + j;
        if (jj >= p.npa) continue;
        // emc_atomic.cu:105-111: divide by the slice's total responsibility
        p.U[r * p.ldU + col_of(p.pix, jj)] = T > 1e-30f ? acc[i][j] / T : acc[i][j];
      }
    }
  }
};

// ----------------------------------------------------------------- softmax --
// 32 patterns per block (lane == pattern), 8 warps share the rotations.  The
// log-likelihood is read from X (FP32, then overwritten by P in place) or, for
// an FP64 log-likelihood, from X64 with P written to X.
template <class T>
__device__ __forceinline__ void softmax_body(const T* L, float* X, int64_t R, int64_t N,
                                             double* plogp_part, double* lse) {
  __shared__ T smax[8][32];
  __shared__ float ssum[8][32];
  __shared__ double sred[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t p = (int64_t)blockIdx.x * 32 + lane;
  const bool ok = p < N;
  T mx = -FLT_MAX;
  if (ok)
    for (int64_t r = w; r < R; r += 8) mx = L[r * N + p] > mx ? L[r * N + p] : mx;
  smax[w][lane] = mx;
  __syncthreads();
  mx = smax[0][lane];
  for (int k = 1; k < 8; ++k) mx = smax[k][lane] > mx ? smax[k][lane] : mx;
  float s = 0.0f;
  if (ok)
    for (int64_t r = w; r < R; r += 8) {
      const float d = (float)(L[r * N + p] - mx);
      if (d > -1.0e10f) s += expf(d);  // emc_cuda.cu:463-468
    }
  ssum[w][lane] = s;
  __syncthreads();
  s = 0.0f;
  for (int k = 0; k < 8; ++k) s += ssum[k][lane];
  const float inv = 1.0f / s;
  if (lse && ok && w == 0) lse[p] = (double)mx + log((double)s);
  double pl = 0.0;
  if (ok)
    for (int64_t r = w; r < R; r += 8) {
      const float d = (float)(L[r * N + p] - mx);
      const float P = d > -1.0e10f ? expf(d) * inv : 0.0f;
      X[r * N + p] = P;
      if (P > 0.0f) pl += (double)P * log((double)P);
    }
  sred[w][lane] = pl;
  __syncthreads();
  if (w == 0) {
    double t = 0;
    for (int k = 0; k < 8; ++k) t += sred[k][lane];
    t = warp_sum(t);
    if (lane == 0 && plogp_part) plogp_part[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(kBlock) softmax_kernel(float* X, int64_t R, int64_t N,
                                                         double* plogp_part, double* lse) {
  softmax_body<float>(X, X, R, N, plogp_part, lse);
}

__global__ void __launch_bounds__(kBlock) softmax64_kernel(const double* L, float* X, int64_t R,
                                                           int64_t N, double* plogp_part,
                                                           double* lse) {
  softmax_body<double>(L, X, R, N, plogp_part, lse);
}

__global__ void xlogx_partial(const float* x, int64_t n, double* part) {
  __shared__ double red[32];
  double s = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float v = x[i];
    if (v > 0.0f) s += (double)v * log((double)v);
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void sum_f64_kernel(const double* x, int64_t n, double* out) {
  __shared__ double red[32];
  double s = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) *out = s;
}

// --------------------------------------------------------------- scaling --
// den_part[blockIdx.y][p] = sum_{r in chunk} P_rp w_r; lane == pattern.
__global__ void __launch_bounds__(kBlock) rowweighted_kernel(const float* P, const double* wr,
                                                             int64_t R, int64_t N, int64_t rchunk,
                                                             double* part) {
  __shared__ double red[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t p = (int64_t)blockIdx.x * 32 + lane;
  const int64_t r0 = (int64_t)blockIdx.y * rchunk, r1 = min(R, r0 + rchunk);
  double s = 0;
  if (p < N)
    for (int64_t r = r0 + w; r < r1; r += 8) s += (double)P[r * N + p] * wr[r];
  red[w][lane] = s;
  __syncthreads();
  if (w == 0 && p < N) {
    double t = 0;
    for (int k = 0; k < 8; ++k) t += red[k][lane];
    part[(int64_t)blockIdx.y * N + p] = t;
  }
}

__global__ void scaling_finish_kernel(const double* num, const double* part, int64_t nparts,
                                      int64_t N, float* scaling) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  double d = 0;
  for (int64_t k = 0; k < nparts; ++k) d += part[k * N + p];
  // emc_cuda.cu:226; a pattern without photons or weight keeps its scale
  if (num[p] > 0.0 && d > 0.0) scaling[p] = (float)(num[p] / d);
}

__global__ void pattern_stats_kernel(const float* K, const int32_t* pix, int64_t N, int64_t npa,
                                     int64_t ldK, int squares, double* num) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= N) return;
  double s = 0;
  for (int64_t j = lane; j < npa; j += 32) {
    const double k = K[p * ldK + col_of(pix, j)];
    s += squares ? k * k : k;
  }
  s = warp_sum(s);
  if (lane == 0) num[p] = s;
}

// best[p] = argmax_r P[r][p] (first on ties), bestv[p] = that value: 32
// patterns per block (lane), the 8 warps split the rotations.
__global__ void __launch_bounds__(256) col_argmax_kernel(const float* P, int64_t R, int64_t N,
                                                         int32_t* best, float* bestv) {
  __shared__ float sv[8][32];
  __shared__ int32_t si[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t p = (int64_t)blockIdx.x * 32 + lane;
  float bv = -INFINITY;
  int32_t bi = -1;
  if (p < N)
    for (int64_t r = w; r < R; r += 8) {
      const float v = P[r * N + p];
      if (v > bv) {
        bv = v;
        bi = (int32_t)r;
      }
    }
  sv[w][lane] = bv;
  si[w][lane] = bi;
  __syncthreads();
  if (w == 0 && p < N) {
    for (int k = 1; k < 8; ++k)
      if (sv[k][lane] > bv || (sv[k][lane] == bv && si[k][lane] >= 0 && si[k][lane] < bi)) {
        bv = sv[k][lane];
        bi = si[k][lane];
      }
    best[p] = bi;
    bestv[p] = bv;
  }
}

__global__ void row_sums_kernel(const float* P, int64_t R, int64_t N, float* T) {
  const int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= R) return;
  double s = 0;
  for (int64_t p = lane; p < N; p += 32) s += P[r * N + p];
  s = warp_sum(s);
  if (lane == 0) T[r] = (float)s;
}

// ----------------------------------------------------------------- insert --
// One block per rotation (emc_atomic.cu:115-133 + :17-73).
__global__ void __launch_bounds__(kBlock) insert_kernel(const InsertArgs a) {
  const int64_t r = blockIdx.x;
  const float T = a.T[r];
  // emc_atomic.cu:128 skips T_r <= 1e-10 (T_r over every pattern shard)
  if (!((a.Tskip ? a.Tskip[r] : T) > 1e-10f) || !(T > 0.0f)) return;
  const float w = a.rotw[r] * T;
  float m[9];
  emc_voxel::rotation_matrix(a.quat + 4 * r, m);
  for (int64_t i = threadIdx.x; i < a.npix; i += blockDim.x) {
    if (a.ins[i] != 1) continue;
    float u[3];
    emc_voxel::position(m, a.side, a.cx[i], a.cy[i], a.cz[i], u);
    const float s = a.U[r * a.ldU + i];
    // FP32 atomics, or the order-independent fixed-point limbs
    auto add = [&](int64_t v, float x, float y) {
      if (a.acc64) {
        add_fixed(a.acc64 + 8 * v, x);
        add_fixed(a.acc64 + 8 * v + 4, y);
      } else {
        atomicAdd(a.model + v, x);
        atomicAdd(a.weight + v, y);
      }
    };
    if (a.interp == 0) {
      int64_t v;
      if (!emc_voxel::nearest(u, a.side, 0, &v)) continue;
      add(v, w * s, w);
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        int64_t v;
        float wc;
        if (!emc_voxel::trilinear_corner(u, a.side, c, &v, &wc) || wc == 0.0f) continue;
        add(v, wc * w * s, wc * w);
      }
    }
  }
}

// ------------------------------------------------------------- normalise --
// Fixed-point accumulators -> FP32 (value, weight) pairs: a[i*stride],
// b[i*stride] (the FP32 path's model and weight, or the mixed path's
// interleaved accumulators), each sum rounded once.
__global__ void fixed_to_pairs_kernel(const unsigned long long* acc64, int64_t M, float* a,
                                      float* b, int64_t stride) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x) {
    a[i * stride] = (float)fixed_value(acc64 + 8 * i);
    b[i * stride] = (float)fixed_value(acc64 + 8 * i + 4);
  }
}

__global__ void divide_kernel(float* model, const float* weight, int64_t M, int fp64,
                              double* part) {
  __shared__ double red[32];
  double s = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float wv = weight[i];
    float v;
    if (wv > 0.0f)  // emc_cuda.cu:416-420
      v = fp64 ? (float)((double)model[i] / (double)wv) : model[i] / wv;
    else
      v = 0.0f;
    model[i] = v;
    s += v;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Mixed path: model/weight from the interleaved accumulators (FP64 division).
__global__ void divide_acc_kernel(const float2* acc, float* model, float* weight, int64_t M,
                                  double* part) {
  __shared__ double red[32];
  double s = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float2 a = acc[i];
    const float v = a.y > 0.0f ? (float)((double)a.x / (double)a.y) : 0.0f;  // emc_cuda.cu:416-420
    model[i] = v;
    weight[i] = a.y;
    s += v;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void scale_max_kernel(float* model, int64_t M, const double* sum, int fp64,
                                 double* stats, double* part) {
  __shared__ float red[32];
  const double mean = *sum / (double)M;
  const float f = (float)(1.0 / mean);
  float mx = 0.0f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (int64_t)gridDim.x * blockDim.x) {
    float v = model[i];
    if (mean != 0.0) v = fp64 ? (float)((double)v / mean) : v * f;
    model[i] = v;
    mx = fmaxf(mx, v);
  }
  mx = block_max(mx, red);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = mx;
    if (blockIdx.x == 0) stats[0] = mean;
  }
}

__global__ void max_partial_kernel(const float* x, int64_t n, double* part) {
  __shared__ float red[32];
  float mx = -FLT_MAX;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    mx = fmaxf(mx, x[i]);
  mx = block_max(mx, red);
  if (threadIdx.x == 0) part[blockIdx.x] = mx;
}

__global__ void max_f64_kernel(const double* x, int64_t n, double* out) {
  __shared__ float red[32];
  float mx = -FLT_MAX;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) mx = fmaxf(mx, (float)x[i]);
  mx = block_max(mx, red);
  if (threadIdx.x == 0) *out = mx;
}

__global__ void fill_kernel(float* x, int64_t n, float v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = v;
}

constexpr int kReduceBlocks = 592;  // 4 x 148 SMs; partial arrays hold this many values

inline int grid_for(int64_t n) {
  const int64_t b = (n + kBlock - 1) / kBlock;
  return (int)(b < kReduceBlocks ? (b > 0 ? b : 1) : kReduceBlocks);
}

}  // namespace

// ------------------------------------------------------------- launchers --

template <int INTERP>
void expand_dispatch(const ExpandArgs& a, cudaStream_t st) {
  if (a.out == EXP_F32)
    expand_kernel<INTERP, EXP_F32><<<(unsigned)a.R, kBlock, 0, st>>>(a);
  else if (a.out == EXP_LOG_F32)
    expand_kernel<INTERP, EXP_LOG_F32><<<(unsigned)a.R, kBlock, 0, st>>>(a);
  else
    expand_kernel<INTERP, EXP_F16_SPLIT><<<(unsigned)a.R, kBlock, 0, st>>>(a);
}

cudaError_t launch_expand(const ExpandArgs& a, cudaStream_t st) {
  if (a.R <= 0) return cudaSuccess;
  if (a.tab && a.interp == 0 && a.out == EXP_F16_SPLIT) {
    if (a.ld % 2 != 0 || a.npix > a.ld || a.ld > (int64_t)1 << 30 || a.stat_mask)
      return cudaErrorInvalidValue;
    expand_tab_kernel<<<(unsigned)a.R, kBlock, 0, st>>>(a);
    return cudaGetLastError();
  }
  if (a.interp == 0)
    expand_dispatch<0>(a, st);
  else
    expand_dispatch<1>(a, st);
  return cudaGetLastError();
}

int64_t tri_table_entries(int side) { return 2 * (int64_t)(side + 1) * (side + 1) * (side + 1); }

cudaError_t launch_tri_table(const float* model, int side, float4* tri, cudaStream_t st) {
  const int64_t n = (int64_t)(side + 1) * (side + 1) * (side + 1);
  tri_table_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(model, side, tri);
  return cudaGetLastError();
}

cudaError_t launch_expand_table(const float* model, int64_t M, float floor_, int log_split,
                                uint2* tab, cudaStream_t st) {
  expand_table_kernel<<<(unsigned)((M + 1 + 255) / 256), 256, 0, st>>>(model, M, floor_, log_split,
                                                                      tab);
  return cudaGetLastError();
}

// ------------------------------------------------------------ photon lists --
// Gathers over the non-zero counts.  One block: 128 threads x 4 rotations =
// 512 rotations by 16 output columns (patterns of the log-likelihood, pixels
// of the slice sums).  For each column the block walks its entries (uniform
// loads of the sparse entry) and every thread gathers 16 bytes of the
// transposed operand row at that entry (logWT[pixel] for the log-likelihood,
// PT[pattern] for the slice sums), so one entry reads one coalesced 2 KB row.
// Column blocks vary fastest in the grid, so the blocks resident at one time
// share one rotation block's columns of the operand in L2.  FP32 partial sums
// over chunks of 32 entries are folded into FP64 totals, as the dense
// contraction folds each 32-wide K-step.  The 16 x 512 results leave through
// shared memory as rows of the output.
//   MODE 0: LL[r][p] = total - phi_p sum W_r      MODE 1: U[r][j] = total / T_r
constexpr int kSparseRot = 512, kSparsePat = 16;
template <int MODE>
__global__ void __launch_bounds__(128)
    sparse_gather_kernel(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                         const float* __restrict__ val, const float* __restrict__ XT,
                         int64_t ldT, int64_t R, int64_t ncol, const float* scaling,
                         const double* rowstat, const float* T, float* out, double* out64) {
  __shared__ float tile[kSparsePat][kSparseRot + 1];
  const int64_t r0 = (int64_t)blockIdx.y * kSparseRot + 4 * threadIdx.x;
  const int64_t p0 = (int64_t)blockIdx.x * kSparsePat;
  const bool rv = r0 < R;  // ldT >= R rounded up to 4: the whole float4 is in bounds
  double sw[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    if (MODE == 0)
      sw[u] = r0 + u < R ? rowstat[r0 + u] : 0.0;
    else
      sw[u] = r0 + u < R ? (double)T[r0 + u] : 0.0;
  }
  for (int i = 0; i < kSparsePat; ++i) {
    const int64_t p = p0 + i;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    if (p < ncol && rv) {
      const int64_t e0 = ptr[p], e1 = ptr[p + 1];
      double tot[4] = {0.0, 0.0, 0.0, 0.0};
      int64_t e = e0;
      while (e < e1) {
        const int64_t ce = e + 32 < e1 ? e + 32 : e1;
        float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0;
        for (; e + 2 <= ce; e += 2) {
          const int32_t j0 = __ldg(idx + e), j1 = __ldg(idx + e + 1);
          const float k0 = __ldg(val + e), k1 = __ldg(val + e + 1);
          const float4 w0 = __ldg(reinterpret_cast<const float4*>(XT + (int64_t)j0 * ldT + r0));
          const float4 w1 = __ldg(reinterpret_cast<const float4*>(XT + (int64_t)j1 * ldT + r0));
          s0.x = fmaf(k0, w0.x, s0.x); s0.y = fmaf(k0, w0.y, s0.y);
          s0.z = fmaf(k0, w0.z, s0.z); s0.w = fmaf(k0, w0.w, s0.w);
          s1.x = fmaf(k1, w1.x, s1.x); s1.y = fmaf(k1, w1.y, s1.y);
          s1.z = fmaf(k1, w1.z, s1.z); s1.w = fmaf(k1, w1.w, s1.w);
        }
        if (e < ce) {
          const float k0 = __ldg(val + e);
          const float4 w0 =
              __ldg(reinterpret_cast<const float4*>(XT + (int64_t)__ldg(idx + e) * ldT + r0));
          s0.x = fmaf(k0, w0.x, s0.x); s0.y = fmaf(k0, w0.y, s0.y);
          s0.z = fmaf(k0, w0.z, s0.z); s0.w = fmaf(k0, w0.w, s0.w);
          ++e;
        }
        tot[0] += (double)(s0.x + s1.x);
        tot[1] += (double)(s0.y + s1.y);
        tot[2] += (double)(s0.z + s1.z);
        tot[3] += (double)(s0.w + s1.w);
      }
      if (MODE == 0) {
        const double ph = (double)scaling[p];
        if (out64) {
          // FP64 results leave from registers (one column of 4 rows each)
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (r0 + u < R) out64[(r0 + u) * ncol + p] = tot[u] - ph * sw[u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = (float)(tot[u] - ph * sw[u]);
      } else {
        // emc_atomic.cu:105-111: divide by the slice's total responsibility
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const float Tr = (float)sw[u];
          v[u] = Tr > 1e-30f ? (float)tot[u] / Tr : (float)tot[u];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) tile[i][4 * threadIdx.x + u] = v[u];
  }
  if (out64) return;  // uniform over the block
  __syncthreads();
  // half a warp per output row: lane & 15 = column
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t p = p0 + (lane & 15);
  for (int rr = 2 * w + (lane >> 4); rr < kSparseRot; rr += 8) {
    const int64_t ro = (int64_t)blockIdx.y * kSparseRot + rr;
    if (ro < R && p < ncol) out[ro * ncol + p] = tile[lane & 15][rr];
  }
}

__global__ void scale_entries_kernel(const float* val, const int32_t* row, const float* scaling,
                                     int64_t nnz, float* out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < nnz) out[e] = val[e] / scaling[row[e]];
}

cudaError_t launch_ll_sparse(const SparseLLArgs& a, cudaStream_t st) {
  if (a.R <= 0 || a.N <= 0) return cudaSuccess;
  if (a.ldT % 4 != 0 || a.ldT < a.R || (reinterpret_cast<uintptr_t>(a.logWT) & 15u))
    return cudaErrorInvalidValue;
  dim3 grid((unsigned)((a.N + kSparsePat - 1) / kSparsePat),
            (unsigned)((a.R + kSparseRot - 1) / kSparseRot));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  sparse_gather_kernel<0><<<grid, 128, 0, st>>>(a.row_ptr, a.col, a.val, a.logWT, a.ldT, a.R, a.N,
                                                a.scaling, a.rowstat, nullptr, a.LL, a.LL64);
  return cudaGetLastError();
}

cudaError_t launch_compress_sparse(const SparseCmpArgs& a, cudaStream_t st) {
  if (a.R <= 0 || a.npa <= 0) return cudaSuccess;
  if (a.ldT % 4 != 0 || a.ldT < a.R || (reinterpret_cast<uintptr_t>(a.PT) & 15u))
    return cudaErrorInvalidValue;
  dim3 grid((unsigned)((a.npa + kSparsePat - 1) / kSparsePat),
            (unsigned)((a.R + kSparseRot - 1) / kSparseRot));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  sparse_gather_kernel<1><<<grid, 128, 0, st>>>(a.col_ptr, a.row, a.val, a.PT, a.ldT, a.R, a.npa,
                                                nullptr, nullptr, a.T, a.U, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_scale_entries(const float* val, const int32_t* row, const float* scaling,
                                 int64_t nnz, float* val_out, cudaStream_t st) {
  if (nnz <= 0) return cudaSuccess;
  scale_entries_kernel<<<(unsigned)((nnz + 255) / 256), 256, 0, st>>>(val, row, scaling, nnz,
                                                                     val_out);
  return cudaGetLastError();
}

__global__ void transpose_kernel(const float* S, int64_t R, int64_t npa, float* ST, int64_t ldT) {
  __shared__ float t[32][33];
  const int64_t j0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t r = r0 + i, j = j0 + threadIdx.x;
    t[i][threadIdx.x] = (r < R && j < npa) ? S[r * npa + j] : 0.0f;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int64_t j = j0 + i, r = r0 + threadIdx.x;
    if (j < npa && r < R) ST[j * ldT + r] = t[threadIdx.x][i];
  }
}

cudaError_t launch_transpose(const float* S, int64_t R, int64_t npa, float* ST, int64_t ldT,
                             cudaStream_t st) {
  dim3 grid((unsigned)((npa + 31) / 32), (unsigned)((R + 31) / 32));
  if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
  transpose_kernel<<<grid, dim3(32, 8), 0, st>>>(S, R, npa, ST, ldT);
  return cudaGetLastError();
}

// one warp per pattern
__global__ void csr_count_kernel(const float* K, int64_t N, int64_t npa, int64_t* count) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= N) return;
  int64_t n = 0;
  for (int64_t j = lane; j < npa; j += 32) n += K[p * npa + j] != 0.0f;
  for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if (lane == 0) count[p] = n;
}

__global__ void csr_fill_kernel(const float* K, int64_t N, int64_t npa, const int64_t* row_ptr,
                                int32_t* col, float* val) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= N) return;
  int64_t out = row_ptr[p];
  for (int64_t j0 = 0; j0 < npa; j0 += 32) {
    const int64_t j = j0 + lane;
    const float k = j < npa ? K[p * npa + j] : 0.0f;
    const unsigned nz = __ballot_sync(0xffffffffu, k != 0.0f);
    if (k != 0.0f) {
      const int64_t o = out + __popc(nz & ((1u << lane) - 1u));
      col[o] = (int32_t)j;
      val[o] = k;
    }
    out += __popc(nz);
  }
}

cudaError_t launch_csr_count(const float* K, int64_t N, int64_t npa, int64_t* count,
                             cudaStream_t st) {
  csr_count_kernel<<<(unsigned)((N + 7) / 8), 256, 0, st>>>(K, N, npa, count);
  return cudaGetLastError();
}

cudaError_t launch_csr_fill(const float* K, int64_t N, int64_t npa, const int64_t* row_ptr,
                            int32_t* col, float* val, cudaStream_t st) {
  csr_fill_kernel<<<(unsigned)((N + 7) / 8), 256, 0, st>>>(K, N, npa, row_ptr, col, val);
  return cudaGetLastError();
}

cudaError_t launch_ll_fp32(const LLArgs& a, cudaStream_t st) {
  if (a.R <= 0 || a.N <= 0) return cudaSuccess;
  dim3 grid((unsigned)((a.N + TN - 1) / TN), (unsigned)((a.R + TM - 1) / TM));
  if (a.poisson) {
    OpLLPoisson op;
    op.p = a;
    tile_kernel<<<grid, kBlock, 0, st>>>(op);
  } else {
    OpLLGauss op;
    op.p = a;
    tile_kernel<<<grid, kBlock, 0, st>>>(op);
  }
  return cudaGetLastError();
}

cudaError_t launch_softmax_from_f64(const double* L, float* P, int64_t R, int64_t N,
                                    double* plogp_part, int* nparts, double* lse,
                                    cudaStream_t st) {
  const int64_t nb = (N + 31) / 32;
  if (nparts) *nparts = (int)nb;
  softmax64_kernel<<<(unsigned)nb, kBlock, 0, st>>>(L, P, R, N, plogp_part, lse);
  return cudaGetLastError();
}

cudaError_t launch_softmax_fp32(float* X, int64_t R, int64_t N, double* plogp_part, int* nparts,
                                double* lse, cudaStream_t st) {
  const int64_t nb = (N + 31) / 32;
  if (nparts) *nparts = (int)nb;
  softmax_kernel<<<(unsigned)nb, kBlock, 0, st>>>(X, R, N, plogp_part, lse);
  return cudaGetLastError();
}

cudaError_t launch_xlogx_sum(const float* x, int64_t n, double* out, double* scratch,
                             cudaStream_t st) {
  const int g = grid_for(n);
  xlogx_partial<<<g, kBlock, 0, st>>>(x, n, scratch);
  sum_f64_kernel<<<1, kBlock, 0, st>>>(scratch, g, out);
  return cudaGetLastError();
}

cudaError_t launch_scaling_cross(const CrossArgs& a, cudaStream_t st) {
  dim3 grid((unsigned)((a.N + TN - 1) / TN), (unsigned)((a.R + TM - 1) / TM));
  OpCross op;
  op.p = a;
  tile_kernel<<<grid, kBlock, 0, st>>>(op);
  return cudaGetLastError();
}

cudaError_t launch_scaling_rowweighted(const float* P, const double* w, int64_t R, int64_t N,
                                       double* den_part, int64_t* nparts, cudaStream_t st) {
  const int64_t rchunk = 1024;
  const int64_t nc = (R + rchunk - 1) / rchunk;
  *nparts = nc;
  dim3 grid((unsigned)((N + 31) / 32), (unsigned)nc);
  rowweighted_kernel<<<grid, kBlock, 0, st>>>(P, w, R, N, rchunk, den_part);
  return cudaGetLastError();
}

cudaError_t launch_scaling_finish(const double* num, const double* den_part, int64_t nparts,
                                  int64_t N, float* scaling, cudaStream_t st) {
  scaling_finish_kernel<<<(unsigned)((N + kBlock - 1) / kBlock), kBlock, 0, st>>>(num, den_part,
                                                                                 nparts, N, scaling);
  return cudaGetLastError();
}

cudaError_t launch_pattern_stats(const float* K, const int32_t* pix, int64_t N, int64_t npa,
                                 int64_t ldK, int squares, double* num, cudaStream_t st) {
  pattern_stats_kernel<<<(unsigned)((N + 7) / 8), kBlock, 0, st>>>(K, pix, N, npa, ldK, squares, num);
  return cudaGetLastError();
}

cudaError_t launch_col_argmax(const float* P, int64_t R, int64_t N, int32_t* best, float* bestv,
                              cudaStream_t st) {
  col_argmax_kernel<<<(unsigned)((N + 31) / 32), 256, 0, st>>>(P, R, N, best, bestv);
  return cudaGetLastError();
}

cudaError_t launch_row_sums(const float* P, int64_t R, int64_t N, float* T, cudaStream_t st) {
  row_sums_kernel<<<(unsigned)((R + 7) / 8), kBlock, 0, st>>>(P, R, N, T);
  return cudaGetLastError();
}

cudaError_t launch_compress_fp32(const CompressArgs& a, cudaStream_t st) {
  dim3 grid((unsigned)((a.npa + TN - 1) / TN), (unsigned)((a.R + TM - 1) / TM));
  OpCompress op;
  op.p = a;
  tile_kernel<<<grid, kBlock, 0, st>>>(op);
  return cudaGetLastError();
}

cudaError_t launch_insert(const InsertArgs& a, cudaStream_t st) {
  if (a.R <= 0) return cudaSuccess;
  insert_kernel<<<(unsigned)a.R, kBlock, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_normalize_model(float* model, const float* weight, int64_t M, int fp64,
                                   double* scratch, double* stats, cudaStream_t st) {
  // scratch: kReduceBlocks + 2 doubles; stats[0] = mean, stats[1] = max
  const int g = grid_for(M);
  divide_kernel<<<g, kBlock, 0, st>>>(model, weight, M, fp64, scratch);
  sum_f64_kernel<<<1, kBlock, 0, st>>>(scratch, g, scratch + kReduceBlocks);
  scale_max_kernel<<<g, kBlock, 0, st>>>(model, M, scratch + kReduceBlocks, fp64, stats, scratch);
  max_f64_kernel<<<1, kBlock, 0, st>>>(scratch, g, stats + 1);
  return cudaGetLastError();
}

cudaError_t launch_fixed_to_pairs(const unsigned long long* acc64, int64_t M, float* a, float* b,
                                  int64_t stride, cudaStream_t st) {
  fixed_to_pairs_kernel<<<grid_for(M), kBlock, 0, st>>>(acc64, M, a, b, stride);
  return cudaGetLastError();
}

cudaError_t launch_normalize_acc(const float2* acc, float* model, float* weight, int64_t M,
                                 double* scratch, double* stats, cudaStream_t st) {
  const int g = grid_for(M);
  divide_acc_kernel<<<g, kBlock, 0, st>>>(acc, model, weight, M, scratch);
  sum_f64_kernel<<<1, kBlock, 0, st>>>(scratch, g, scratch + kReduceBlocks);
  scale_max_kernel<<<g, kBlock, 0, st>>>(model, M, scratch + kReduceBlocks, 1, stats, scratch);
  max_f64_kernel<<<1, kBlock, 0, st>>>(scratch, g, stats + 1);
  return cudaGetLastError();
}

cudaError_t launch_model_max(const float* model, int64_t M, double* scratch, double* out,
                             cudaStream_t st) {
  const int g = grid_for(M);
  max_partial_kernel<<<g, kBlock, 0, st>>>(model, M, scratch);
  max_f64_kernel<<<1, kBlock, 0, st>>>(scratch, g, out);
  return cudaGetLastError();
}

cudaError_t launch_fill(float* x, int64_t n, float v, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  fill_kernel<<<grid_for(n), kBlock, 0, st>>>(x, n, v);
  return cudaGetLastError();
}

__global__ void count_invalid_kernel(const float* x, int64_t n, int* bad) {
  int nb = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float v = x[i];
    if (!(v >= 0.0f && v <= FLT_MAX)) nb++;  // negative, NaN or infinite
  }
  if (nb) atomicAdd(bad, nb);
}

cudaError_t launch_count_invalid(const float* x, int64_t n, int* bad, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  count_invalid_kernel<<<grid_for(n), kBlock, 0, st>>>(x, n, bad);
  return cudaGetLastError();
}

cudaError_t launch_sum_f64(const double* x, int64_t n, double* out, cudaStream_t st) {
  sum_f64_kernel<<<1, kBlock, 0, st>>>(x, n, out);
  return cudaGetLastError();
}

}  // namespace emc
