// Learned rotation proposal: the kernels that connect the proposal network to
// the EMC iteration.
//   features   2x-downsampled log(1 + K) of every pattern (network input)
//   targets    dense responsibilities summed over each coarse cell (training labels)
//   select     the top cells of every pattern's predicted cell posterior
//   grouped    maximize and compress restricted to the fine rotations of the
//              selected cells, one contraction per coarse cell (the patterns
//              that selected the cell x the cell's fine rotations, which are
//              contiguous because the rotation list is sorted by cell)
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "proposal.cuh"
#include "tile.cuh"

namespace emc {
namespace {

__global__ void features_kernel(const float* K, const int32_t* pix, int64_t N, int64_t npa, int side,
                                int S, float* x) {
  const int64_t total = N * npa;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = e / npa, j = e - p * npa;
    const float k = K[e];
    if (k == 0.0f) continue;
    const int i = pix[j], iy = i / side, ix = i % side;
    // integer counts: the sums are exact, so the atomic order does not matter
    atomicAdd(x + p * S * S + (iy / 2) * S + ix / 2, k);
  }
}

__global__ void log1p_kernel(float* x, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = log1pf(x[i]);
}

__device__ __forceinline__ float resp_of(const TargetArgs& a, int64_t r, int64_t p) {
  if (a.P) return a.P[r * a.ldP + p];
  const float y = a.Y[r * a.ldY + p];
  double ll;
  if (a.poisson) {
    ll = (double)y;
  } else {
    const double phi = a.scaling[p];
    ll = ((double)y * 2.0 / phi - a.rowstat[r] - a.patstat[p] / (phi * phi)) * a.gauss_inv;
  }
  return expf((float)(ll - a.lse[p]));
}

// t[p][c] = sum over the fine rotations r of cell c of P_rp; 32 patterns per
// block (lane = pattern), the 8 warps share the rotations, shared-memory sums.
__global__ void __launch_bounds__(256) targets_kernel(const TargetArgs a) {
  extern __shared__ float tc[];  // [n_cells][32]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t p = (int64_t)blockIdx.x * 32 + lane;
  for (int i = threadIdx.x; i < a.n_cells * 32; i += blockDim.x) tc[i] = 0.0f;
  __syncthreads();
  if (p < a.N)
    for (int64_t r = w; r < a.R; r += 8) atomicAdd(&tc[a.cell[r] * 32 + lane], resp_of(a, r, p));
  __syncthreads();
  if (p < a.N)
    for (int c = w; c < a.n_cells; c += 8) a.t[p * a.n_cells + c] = tc[c * 32 + lane];
}

// One warp per pattern: the m most probable cells, and their total probability.
__global__ void select_kernel(const float* probs, int64_t N, int C, int m, int32_t* cand,
                              float* mass) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= N) return;
  const float* row = probs + p * C;
  uint32_t taken = 0;  // bit i: cell lane + 32 i already selected (C <= 1024)
  float tot = 0.0f;
  for (int s = 0; s < m; ++s) {
    float best = -1.0f;
    int bi = -1;
    for (int i = 0; lane + 32 * i < C; ++i) {
      const float v = row[lane + 32 * i];
      if (!((taken >> i) & 1u) && v > best) {
        best = v;
        bi = lane + 32 * i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi >= 0 && (bi < 0 || oi < bi))) {
        best = ov;
        bi = oi;
      }
    }
    if (bi >= 0 && (bi & 31) == lane) taken |= 1u << (bi >> 5);
    if (lane == 0) cand[p * m + s] = bi;
    tot += best > 0.0f ? best : 0.0f;
  }
  if (lane == 0) mass[p] = tot;
}

// Grouped maximize, one contraction per cell (blockIdx.z): rows = the cell's
// fine rotations, columns = its (pattern, cell) pairs, reduction over pixels.
// Writes Y[pair][member]: poisson LL, gaussian cross term C.
struct OpGroupLL {
  using Acc = double;
  static constexpr bool kBKMajor = true;
  GroupArgs g;
  __device__ int64_t ksize() const { return g.npa; }
  __device__ float a(int64_t row, int64_t j) const {
    const int c = blockIdx.z;
    if (row >= g.mcnt[c] || j >= g.npa) return 0.0f;
    const int64_t r = g.mbeg[c] + row;
    if (g.S) return __ldg(g.S + r * g.ldS + j);
    return __half2float(g.hi[r * g.ldS + j]) + __half2float(g.lo[r * g.ldS + j]);
  }
  __device__ float b(int64_t col, int64_t j) const {
    const int c = blockIdx.z;
    if (col >= g.gcnt[c] || j >= g.npa) return 0.0f;
    return __ldg(g.K + (int64_t)g.gpair[g.gbeg[c] + col] * g.npa + j);
  }
  static __device__ __forceinline__ float inner(float acc, float a, float b) { return fmaf(a, b, acc); }
  __device__ void epilogue(double (&acc)[8][4], int64_t r0, int64_t n0, float*) const {
    const int c = blockIdx.z;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int64_t row = r0 + i;
      if (row >= g.mcnt[c]) continue;
      const int64_t r = g.mbeg[c] + row;
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int64_t col = n0 + jj;
        if (col >= g.gcnt[c]) continue;
        const int64_t q = g.gbeg[c] + col;
        const int p = g.gpair[q];
        const double v = g.poisson ? acc[i][jj] - (double)g.scaling[p] * g.rowstat[r] : acc[i][jj];
        g.Y[q * g.MM + row] = (float)v;
      }
    }
  }
};

// Per pattern (one warp): log-sum-exp over its candidate rotations (FP64), new
// scaling, sum P log P; writes P / phi_new into the per-cell compress operand
// Pt and adds P into T_r.
__global__ void group_softmax_kernel(const GroupArgs g) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= g.N) return;
  const double phi = g.scaling[p];
  const double c1 = 2.0 * g.gauss_inv / phi, c0 = g.poisson ? 0.0 : -g.patstat[p] / (phi * phi) * g.gauss_inv;
  auto ll_of = [&](int c, int64_t q, int k) -> double {
    const float y = g.Y[q * g.MM + k];
    if (g.poisson) return (double)y;
    return fma((double)y, c1, c0 - g.rowstat[g.mbeg[c] + k] * g.gauss_inv);
  };
  double mx = -INFINITY;
  for (int i = 0; i < g.m; ++i) {
    const int c = g.cand[p * g.m + i];
    const int64_t q = g.ppos[p * g.m + i];
    for (int k = lane; k < g.mcnt[c]; k += 32) mx = fmax(mx, ll_of(c, q, k));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  double s = 0.0, d = 0.0, pl = 0.0;
  for (int i = 0; i < g.m; ++i) {
    const int c = g.cand[p * g.m + i];
    const int64_t q = g.ppos[p * g.m + i];
    for (int k = lane; k < g.mcnt[c]; k += 32) {
      const double l = ll_of(c, q, k);
      const double e = exp(l - mx);
      s += e;
      d += e * (g.poisson ? g.rowstat[g.mbeg[c] + k] : (double)g.Y[q * g.MM + k]);
      pl += e * (l - mx);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    d += __shfl_xor_sync(0xffffffffu, d, o);
    pl += __shfl_xor_sync(0xffffffffu, pl, o);
  }
  const double lse = mx + log(s);
  // emc_cuda.cu:226 (gaussian) / poisson MLE, over the evaluated rotations
  const double num = g.poisson ? g.patsum[p] : g.patstat[p];
  const double den = d / s;
  const double phi_new = (num > 0.0 && den > 0.0) ? num / den : phi;
  if (lane == 0) {
    g.lse[p] = lse;
    g.plogp[p] = pl / s - log(s);
    g.new_scaling[p] = (float)phi_new;
  }
  for (int i = 0; i < g.m; ++i) {
    const int c = g.cand[p * g.m + i];
    const int64_t q = g.ppos[p * g.m + i];
    const int64_t col = q - g.gbeg[c];
    for (int k = lane; k < g.mcnt[c]; k += 32) {
      const float P = (float)exp(ll_of(c, q, k) - lse);
      g.Pt[g.goff[c] + (int64_t)k * g.gcnt[c] + col] = (float)(P / phi_new);
      atomicAdd(g.T + g.mbeg[c] + k, P);
    }
  }
}

// Grouped compress, one contraction per cell: rows = the cell's rotations,
// columns = pixels, reduction over the cell's pairs: U_r / T_r.
struct OpGroupCmp {
  using Acc = float;
  static constexpr bool kBKMajor = false;
  GroupArgs g;
  __device__ int64_t ksize() const { return g.gcnt[blockIdx.z]; }
  __device__ float a(int64_t row, int64_t k) const {
    const int c = blockIdx.z;
    if (row >= g.mcnt[c] || k >= g.gcnt[c]) return 0.0f;
    return g.Pt[g.goff[c] + row * g.gcnt[c] + k];
  }
  __device__ float b(int64_t j, int64_t k) const {
    const int c = blockIdx.z;
    if (j >= g.npa || k >= g.gcnt[c]) return 0.0f;
    return __ldg(g.K + (int64_t)g.gpair[g.gbeg[c] + k] * g.npa + j);
  }
  static __device__ __forceinline__ float inner(float acc, float a, float b) { return fmaf(a, b, acc); }
  __device__ void epilogue(float (&acc)[8][4], int64_t r0, int64_t j0, float*) const {
    const int c = blockIdx.z;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int64_t row = r0 + i;
      if (row >= g.mcnt[c]) continue;
      const int64_t r = g.mbeg[c] + row;
      const float T = g.T[r];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int64_t j = j0 + jj;
        if (j >= g.npa) continue;
        g.U[r * g.npa + j] = T > 1e-10f ? acc[i][jj] / T : acc[i][jj];
      }
    }
  }
};

inline unsigned blocks_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b < 8192 ? (b > 0 ? b : 1) : 8192);
}

}  // namespace

cudaError_t launch_features(const float* K, const int32_t* pix, int64_t N, int64_t npa, int side,
                            int S, float* x, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(x, 0, sizeof(float) * N * S * S, st);
  if (e != cudaSuccess) return e;
  features_kernel<<<blocks_for(N * npa), 256, 0, st>>>(K, pix, N, npa, side, S, x);
  log1p_kernel<<<blocks_for(N * S * S), 256, 0, st>>>(x, N * S * S);
  return cudaGetLastError();
}

cudaError_t launch_targets(const TargetArgs& a, cudaStream_t st) {
  const size_t smem = sizeof(float) * 32 * a.n_cells;
  cudaError_t e = cudaFuncSetAttribute(targets_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  targets_kernel<<<(unsigned)((a.N + 31) / 32), 256, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_select(const float* probs, int64_t N, int C, int m, int32_t* cand, float* mass,
                          cudaStream_t st) {
  select_kernel<<<(unsigned)((N + 7) / 8), 256, 0, st>>>(probs, N, C, m, cand, mass);
  return cudaGetLastError();
}

cudaError_t launch_group_maximize(const GroupArgs& g, int64_t max_pairs, int64_t max_members,
                                  cudaStream_t st) {
  OpGroupLL op{g};
  dim3 grid((unsigned)((max_pairs + TN - 1) / TN), (unsigned)((max_members + TM - 1) / TM),
            (unsigned)g.n_cells);
  tile_kernel<<<grid, kTileThreads, 0, st>>>(op);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  group_softmax_kernel<<<(unsigned)((g.N + 7) / 8), 256, 0, st>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_group_compress(const GroupArgs& g, int64_t max_members, cudaStream_t st) {
  OpGroupCmp op{g};
  dim3 grid((unsigned)((g.npa + TN - 1) / TN), (unsigned)((max_members + TM - 1) / TM),
            (unsigned)g.n_cells);
  tile_kernel<<<grid, kTileThreads, 0, st>>>(op);
  return cudaGetLastError();
}

}  // namespace emc
