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

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "proposal.cuh"
#include "tile.cuh"
#include "voxel.h"

namespace emc {
namespace {

__device__ __forceinline__ void red_add_v2(float2* p, float x, float y) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(x), "f"(y) : "memory");
}

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

// The cell sums read Y (or P / LL64) once, 32 patterns per block (lane =
// pattern, 128-byte rows) and one cell per warp: the rotations are sorted by
// cell, so a cell is the row range mbeg .. mbeg + mcnt - 1 and each (pattern,
// cell) sum has one owner (no atomics).  Rows are loaded four at a time so
// each warp keeps four loads in flight.
constexpr int kCellWarps = 8;

// t[p][c] = sum over the fine rotations r of cell c of P_rp.
__global__ void __launch_bounds__(256) targets_kernel(const TargetArgs a) {
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.y * kCellWarps + (threadIdx.x >> 5);
  const int64_t p = (int64_t)blockIdx.x * 32 + lane;
  if (c >= a.n_cells || p >= a.N) return;
  const int64_t r0 = a.mbeg[c], r1 = r0 + a.mcnt[c];
  float sum = 0.0f;
  for (int64_t r = r0; r < r1; r += 4) {
    float v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = r + u < r1 ? resp_of(a, r + u, p) : 0.0f;
    sum += (v[0] + v[1]) + (v[2] + v[3]);
  }
  a.t[p * a.n_cells + c] = sum;
}

// lt[p][c] = natural log of the responsibility mass of cell c in the log
// domain (an online maximum with a rescaled FP64 sum of exponentials), so
// every cell is ranked however far down the tail it lies.  Layout as
// targets_kernel.
__global__ void __launch_bounds__(256) log_targets_kernel(const TargetArgs a) {
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.y * kCellWarps + (threadIdx.x >> 5);
  const int64_t p = (int64_t)blockIdx.x * 32 + lane;
  if (c >= a.n_cells || p >= a.N) return;
  auto ll_of = [&](int64_t r) -> double {  // log-likelihood (FP32 path: minus lse)
    if (a.L64) return a.L64[r * a.ldP + p];
    if (a.P) return log((double)a.P[r * a.ldP + p]);
    const float y = a.Y[r * a.ldY + p];
    if (a.poisson) return (double)y;
    const double phi = a.scaling[p];
    return ((double)y * 2.0 / phi - a.rowstat[r] - a.patstat[p] / (phi * phi)) * a.gauss_inv;
  };
  const double lse = a.P ? 0.0 : a.lse[p];
  const int64_t r0 = a.mbeg[c], r1 = r0 + a.mcnt[c];
  double mx = -INFINITY, sum = 0.0;
  for (int64_t r = r0; r < r1; r += 4) {
    double l[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) l[u] = r + u < r1 ? ll_of(r + u) : -INFINITY;
    // FP64 differences and sum, FP32 exponentials (relative error ~1e-7 in a
    // logarithm that only ranks the cells)
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (!(l[u] > -INFINITY)) continue;
      if (l[u] > mx) {
        sum = sum * (double)expf((float)(mx - l[u])) + 1.0;
        mx = l[u];
      } else {
        sum += (double)expf((float)(l[u] - mx));
      }
    }
  }
  a.t[p * a.n_cells + c] = (sum > 0.0 && mx > -INFINITY) ? (float)(mx + log(sum) - lse) : -INFINITY;
}

// Most probable cell of a row among those not yet taken (lane owns cells
// lane + 32 i, bit i of `taken`), the lowest index among equals; bi = -1 when
// every remaining value is NaN.
__device__ __forceinline__ void warp_argmax(const float* row, int C, uint32_t taken, int lane,
                                            float& best, int& bi) {
  best = -INFINITY;
  bi = -1;
  for (int i = 0; lane + 32 * i < C; ++i) {
    const float v = row[lane + 32 * i];
    if (!((taken >> i) & 1u) && (v > best || (bi < 0 && v == v))) {
      best = v;
      bi = lane + 32 * i;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (oi >= 0 && (bi < 0 || ov > best || (ov == best && oi < bi))) {
      best = ov;
      bi = oi;
    }
  }
}

// One warp per pattern.  With `keep`: first its most probable cells under
// keep (those with keep > 0) until at least min_m are taken and their keep
// total reaches keep_mass.  Then cells in order of probs until at least min_m
// are taken and their probs total reaches mass_target, at most m; unused
// slots -1.  mass[p] = the probs total of the taken cells.
__global__ void select_kernel(const float* probs, const float* keep, int64_t N, int C, int min_m,
                              int m, float mass_target, float keep_mass, int32_t* cand,
                              float* mass) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= N) return;
  const float* row = probs + p * C;
  uint32_t taken = 0;  // bit i: cell lane + 32 i already selected (C <= 1024)
  float tot = 0.0f;
  const bool adaptive = mass_target < 1.0f;  // else always m cells
  int s = 0;
  if (keep) {
    const float* krow = keep + p * C;
    float ktot = 0.0f;
    for (; s < m && (s < min_m || ktot < keep_mass); ++s) {
      float best;
      int bi;
      warp_argmax(krow, C, taken, lane, best, bi);
      if (bi < 0 || !(best > 0.0f)) break;
      ktot += best;
      if ((bi & 31) == lane) taken |= 1u << (bi >> 5);
      if (lane == 0) cand[p * m + s] = bi;
      const float v = row[bi];
      tot += v > 0.0f ? v : 0.0f;
    }
  }
  for (; s < m && !(adaptive && s >= min_m && tot >= mass_target); ++s) {
    float best;
    int bi;
    warp_argmax(row, C, taken, lane, best, bi);
    if (bi >= 0 && (bi & 31) == lane) taken |= 1u << (bi >> 5);
    if (lane == 0) cand[p * m + s] = bi;
    tot += best > 0.0f ? best : 0.0f;
  }
  for (int k = s + lane; k < m; k += 32) cand[p * m + k] = -1;
  if (lane == 0) mass[p] = tot;
}

// Top-k selection, one warp per pattern.  With log_keep (the log-posterior
// mass of every cell in a previous iteration): cells in order of it (finite
// values only) until they hold at least top_k fine rotations and, with
// keep_tail > 0, all but keep_tail of that posterior.  Then, with
// probs (a predicted cell posterior): cells in order of probs until the probs
// total of everything taken reaches mass_target.  At most m cells; unused
// slots -1; mass[p] = the probs total of the taken cells (1 without probs).
__global__ void select_topk_kernel(const float* probs, const float* log_keep, const int32_t* mcnt,
                                   int64_t N, int C, int top_k, int m, float mass_target,
                                   float keep_tail, int32_t* cand, float* mass) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= N) return;
  uint32_t taken = 0;  // bit i: cell lane + 32 i already selected (C <= 1024)
  float tot = 0.0f;
  int s = 0;
  if (log_keep) {
    const float* krow = log_keep + p * C;
    int64_t covered = 0;
    double held = 0.0;  // previous posterior mass of the taken cells
    for (; s < m && (covered < top_k || (keep_tail > 0.0f && held < 1.0 - keep_tail)); ++s) {
      float best;
      int bi;
      warp_argmax(krow, C, taken, lane, best, bi);
      if (bi < 0 || !(best > -INFINITY)) break;
      if ((bi & 31) == lane) taken |= 1u << (bi >> 5);
      if (lane == 0) cand[p * m + s] = bi;
      covered += mcnt[bi];
      held += exp((double)best);
      if (probs) {
        const float v = probs[p * C + bi];
        tot += v > 0.0f ? v : 0.0f;
      }
    }
  }
  if (probs) {
    const float* row = probs + p * C;
    for (; s < m && (s == 0 || tot < mass_target); ++s) {
      float best;
      int bi;
      warp_argmax(row, C, taken, lane, best, bi);
      if (bi < 0) break;
      if ((bi & 31) == lane) taken |= 1u << (bi >> 5);
      if (lane == 0) cand[p * m + s] = bi;
      tot += best > 0.0f ? best : 0.0f;
    }
  }
  for (int k = s + lane; k < m; k += 32) cand[p * m + k] = -1;
  if (lane == 0) mass[p] = probs ? tot : 1.0f;
}

// Dense audit of a sample of patterns: for audited pattern a (global index
// pat[a]) the share of its responsibility that falls on the fine rotations of
// its candidate cells, from its log-likelihood against every rotation:
// LL64 [R][ld] (FP64) or the mixed path's Y [R][ld] (poisson LL, gaussian
// cross term C).  One block per audited pattern.
__global__ void __launch_bounds__(256) audit_kernel(const AuditArgs a) {
  __shared__ uint32_t mask[32];  // candidate cells (n_cells <= 1024)
  __shared__ double red[8];
  const int aidx = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int64_t p = a.pat[aidx];
  if (t < 32) mask[t] = 0u;
  __syncthreads();
  for (int i = t; i < a.m; i += blockDim.x) {
    const int c = a.cand[p * a.m + i];
    if (c >= 0) atomicOr(&mask[c >> 5], 1u << (c & 31));
  }
  __syncthreads();
  const double phi = a.scaling ? (double)a.scaling[aidx] : 1.0;
  auto ll_of = [&](int64_t r) -> double {
    if (a.LL64) return a.LL64[r * a.ld + aidx];
    const double y = (double)a.Y[r * a.ld + aidx];
    if (a.poisson) return y;
    return (y * 2.0 / phi - a.rowstat[r] - a.patstat[aidx] / (phi * phi)) * a.gauss_inv;
  };
  double mx = -INFINITY;
  for (int64_t r = t; r < a.R; r += blockDim.x) mx = fmax(mx, ll_of(r));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) red[w] = mx;
  __syncthreads();
  mx = red[0];
  for (int k = 1; k < 8; ++k) mx = fmax(mx, red[k]);
  __syncthreads();
  double s = 0.0, in = 0.0;
  for (int64_t r = t; r < a.R; r += blockDim.x) {
    const double e = (double)expf((float)(ll_of(r) - mx));
    s += e;
    const int c = a.cell[r];
    if ((mask[c >> 5] >> (c & 31)) & 1u) in += e;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    in += __shfl_xor_sync(0xffffffffu, in, o);
  }
  __shared__ double red2[8];
  if (lane == 0) {
    red[w] = s;
    red2[w] = in;
  }
  __syncthreads();
  if (t == 0) {
    double S = 0.0, I = 0.0;
    for (int k = 0; k < 8; ++k) {
      S += red[k];
      I += red2[k];
    }
    a.captured[aidx] = (float)(I / S);
  }
}

// FP32 responsibilities [R][N] of a proposed iteration (0 outside each
// pattern's candidate cells; P zeroed by the caller): one warp per pattern.
__global__ void proposed_resp_kernel(const GroupArgs g, float* P) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= g.N) return;
  const double phi = g.scaling[p];
  const double c1 = 2.0 * g.gauss_inv / phi,
               c0 = g.poisson ? 0.0 : -g.patstat[p] / (phi * phi) * g.gauss_inv;
  const double lse = g.lse[p];
  for (int i = 0; i < g.m; ++i) {
    const int c = g.cand[p * g.m + i];
    if (c < 0) break;
    const int64_t q = g.ppos[p * g.m + i];
    for (int k = lane; k < g.mcnt[c]; k += 32) {
      const double y = (double)g.Y[q * g.MM + k];
      const double l = g.poisson ? y : fma(y, c1, c0 - g.rowstat[g.mbeg[c] + k] * g.gauss_inv);
      P[(g.mbeg[c] + k) * g.N + p] = (float)exp(l - lse);
    }
  }
}

// Grouped maximize, one contraction per cell: rows = the cell's fine
// rotations, columns = its (pattern, cell) pairs, reduction over pixels.
// Blocks come from a tile list (cell, row offset, column offset) holding only
// the tiles of cells that some pattern selected.  Writes Y[pair][member]:
// poisson LL, gaussian cross term.
struct OpGroupLL {
  using Acc = double;
  static constexpr bool kBKMajor = true;
  GroupArgs g;
  __device__ int cell() const { return __ldg(&g.mtiles[blockIdx.x].x); }
  __device__ bool origin(int64_t& m0, int64_t& n0) const {
    const int4 t = g.mtiles[blockIdx.x];
    m0 = t.y;
    n0 = t.z;
    return true;
  }
  __device__ int64_t ksize() const { return g.npa; }
  __device__ float a(int64_t row, int64_t j) const {
    const int c = cell();
    if (row >= __ldg(g.mcnt + c) || j >= g.npa) return 0.0f;
    const int64_t r = __ldg(g.mbeg + c) + row;
    if (g.S) return __ldg(g.S + r * g.ldS + j);
    return __half2float(g.hi[r * g.ldS + j]) + __half2float(g.lo[r * g.ldS + j]);
  }
  __device__ float b(int64_t col, int64_t j) const {
    const int c = cell();
    if (col >= __ldg(g.gcnt + c) || j >= g.npa) return 0.0f;
    return __ldg(g.K + (int64_t)__ldg(g.gpair + __ldg(g.gbeg + c) + col) * g.npa + j);
  }
  static __device__ __forceinline__ float inner(float acc, float a, float b) { return fmaf(a, b, acc); }
  __device__ void epilogue(double (&acc)[8][4], int64_t r0, int64_t n0, float*) const {
    const int c = cell();
    const int32_t mc = g.mcnt[c], gc = g.gcnt[c];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int64_t row = r0 + i;
      if (row >= mc) continue;
      const int64_t r = g.mbeg[c] + row;
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int64_t col = n0 + jj;
        if (col >= gc) continue;
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
// Pt (when the grouped compress reads it) and adds P into T_r.
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
  int64_t arg = -1;  // rotation of the largest LL (first in candidate order on ties)
  for (int i = 0; i < g.m; ++i) {
    const int c = g.cand[p * g.m + i];
    if (c < 0) break;
    const int64_t q = g.ppos[p * g.m + i];
    for (int k = lane; k < g.mcnt[c]; k += 32) {
      const double l = ll_of(c, q, k);
      if (l > mx) {
        mx = l;
        arg = g.mbeg[c] + k;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double om = __shfl_xor_sync(0xffffffffu, mx, o);
    const long long oa = __shfl_xor_sync(0xffffffffu, (long long)arg, o);
    if (om > mx || (om == mx && oa >= 0 && (arg < 0 || oa < arg))) {
      mx = om;
      arg = oa;
    }
  }
  double s = 0.0, d = 0.0, pl = 0.0;
  for (int i = 0; i < g.m; ++i) {
    const int c = g.cand[p * g.m + i];
    if (c < 0) break;
    const int64_t q = g.ppos[p * g.m + i];
    for (int k = lane; k < g.mcnt[c]; k += 32) {
      const double l = ll_of(c, q, k);
      // the difference in FP64, exp in FP32 (relative error ~1e-7), sums in FP64
      const double e = (double)expf((float)(l - mx));
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
    g.best_rot[p] = (int32_t)arg;
    g.best_p[p] = (float)exp(mx - lse);
  }
  for (int i = 0; i < g.m; ++i) {
    const int c = g.cand[p * g.m + i];
    if (c < 0) break;
    const int64_t q = g.ppos[p * g.m + i];
    const int64_t col = q - g.gbeg[c];
    // the cell's mass in the log domain (its largest LL, then the sum
    // relative to it), so cells far down the tail are still ranked
    double cmx = -INFINITY;
    if (g.lcmass) {
      for (int k = lane; k < g.mcnt[c]; k += 32) cmx = fmax(cmx, ll_of(c, q, k));
      for (int o = 16; o > 0; o >>= 1) cmx = fmax(cmx, __shfl_xor_sync(0xffffffffu, cmx, o));
    }
    float cm = 0.0f;
    double crel = 0.0;
    for (int k = lane; k < g.mcnt[c]; k += 32) {
      const double l = ll_of(c, q, k);
      const float P = expf((float)(l - lse));
      if (g.Pt) g.Pt[g.goff[c] + (int64_t)k * g.gcnt[c] + col] = (float)(P / phi_new);
      // most candidates of a sharp posterior underflow: no atomic for those
      if (P != 0.0f) atomicAdd(g.T + g.mbeg[c] + k, P);
      cm += P;
      if (g.lcmass) crel += (double)expf((float)(l - cmx));
    }
    for (int o = 16; o > 0; o >>= 1) {
      cm += __shfl_xor_sync(0xffffffffu, cm, o);
      crel += __shfl_xor_sync(0xffffffffu, crel, o);
    }
    if (lane == 0) {
      g.cmass[p * g.m + i] = cm;
      if (g.lcmass)
        g.lcmass[p * g.m + i] =
            (crel > 0.0 && cmx > -INFINITY) ? (float)(cmx + log(crel) - lse) : -INFINITY;
    }
  }
}

// Responsibility lists of a proposed iteration (after the grouped softmax,
// with T_r and the new scaling final): per rotation the patterns whose P is
// at least theta T_r, with x = P / (T_r phi_new).  FILL = 0 counts per rotation
// (cnt [R], zeroed by the caller); FILL = 1 writes the entries at rowoff[r]
// plus a per-rotation cursor (zeroed), in no fixed order within a row.  One
// warp per pattern.
template <int FILL>
__global__ void group_list_kernel(const GroupArgs g, float theta, unsigned long long* cnt,
                                  const int64_t* rowoff, int32_t* pat, float* xv) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= g.N) return;
  const double phi = g.scaling[p];
  const double c1 = 2.0 * g.gauss_inv / phi,
               c0 = g.poisson ? 0.0 : -g.patstat[p] / (phi * phi) * g.gauss_inv;
  const double lse = g.lse[p];
  const float inv_phi = 1.0f / g.new_scaling[p];
  for (int i = 0; i < g.m; ++i) {
    const int c = g.cand[p * g.m + i];
    if (c < 0) break;
    const int64_t q = g.ppos[p * g.m + i];
    for (int k = lane; k < g.mcnt[c]; k += 32) {
      const int64_t r = g.mbeg[c] + k;
      const float T = g.T[r];
      if (!(T > 0.0f)) continue;
      const double y = (double)g.Y[q * g.MM + k];
      const double l = g.poisson ? y : fma(y, c1, c0 - g.rowstat[r] * g.gauss_inv);
      const float P = expf((float)(l - lse));  // as group_softmax_kernel forms it
      if (!(P >= theta * T)) continue;
      const float x = P / T * inv_phi;
      if (FILL == 0) {
        atomicAdd(cnt + r, 1ull);
      } else {
        const int64_t pos = rowoff[r] + (int64_t)atomicAdd(cnt + r, 1ull);
        pat[pos] = (int32_t)p;
        xv[pos] = x;
      }
    }
  }
}

// t[p][c] from a proposed iteration: the responsibility mass of each
// candidate cell, 0 elsewhere (t zeroed by the caller).
__global__ void scatter_targets_kernel(const int32_t* cand, const float* cmass, int64_t N, int m,
                                       int n_cells, float* t) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= N * m) return;
  const int c = cand[e];
  if (c >= 0) t[(e / m) * n_cells + c] = cmass[e];
}

// Grouped compress, one contraction per cell: rows = the cell's rotations,
// columns = pixels, reduction over the cell's pairs, giving T_r U_r; the
// epilogue inserts it into the interleaved (model, weight) accumulators
// (emc_atomic.cu:115-133: weight w = rotw T_r, so model += rotw (T_r U_r)),
// skipping rotations with T_r <= 1e-10.  blockIdx.x indexes the (cell, row
// offset) list, blockIdx.y the pixel tile.
struct OpGroupCmp {
  using Acc = float;
  static constexpr bool kBKMajor = false;
  GroupArgs g;
  __device__ int cell() const { return __ldg(&g.ctiles[blockIdx.x].x); }
  __device__ bool origin(int64_t& m0, int64_t& n0) const {
    m0 = g.ctiles[blockIdx.x].y;
    n0 = (int64_t)blockIdx.y * TN;
    return true;
  }
  __device__ int64_t ksize() const { return g.gcnt[cell()]; }
  __device__ float a(int64_t row, int64_t k) const {
    const int c = cell();
    const int32_t gc = __ldg(g.gcnt + c);
    if (row >= __ldg(g.mcnt + c) || k >= gc) return 0.0f;
    return g.Pt[__ldg(g.goff + c) + row * gc + k];
  }
  __device__ float b(int64_t j, int64_t k) const {
    const int c = cell();
    if (j >= g.npa || k >= __ldg(g.gcnt + c)) return 0.0f;
    return __ldg(g.K + (int64_t)__ldg(g.gpair + __ldg(g.gbeg + c) + k) * g.npa + j);
  }
  static __device__ __forceinline__ float inner(float acc, float a, float b) { return fmaf(a, b, acc); }
  __device__ void epilogue(float (&acc)[8][4], int64_t r0, int64_t j0, float*) const {
    const int c = cell();
    const int32_t mc = g.mcnt[c];
    float cx[4], cy[4], cz[4];
    bool use[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int64_t j = j0 + jj;
      use[jj] = j < g.npa && g.ins[j] == 1;
      cx[jj] = use[jj] ? g.cx[j] : 0.0f;
      cy[jj] = use[jj] ? g.cy[j] : 0.0f;
      cz[jj] = use[jj] ? g.cz[j] : 0.0f;
    }
#pragma unroll 1
    for (int i = 0; i < 8; ++i) {
      const int64_t row = r0 + i;
      if (row >= mc) break;
      const int64_t r = g.mbeg[c] + row;
      const float T = g.T[r];
      if (!(T > 1e-10f)) continue;
      const float rw = g.rotw[r], wT = rw * T;
      float m[9];
      emc_voxel::rotation_matrix(g.quat + 4 * r, m);
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        if (!use[jj]) continue;
        float u[3];
        emc_voxel::position(m, g.side, cx[jj], cy[jj], cz[jj], u);
        const float val = rw * acc[i][jj];
        if (g.interp == 0) {
          int64_t v;
          if (emc_voxel::nearest(u, g.side, 0, &v)) red_add_v2(g.acc + v, val, wT);
        } else {
#pragma unroll
          for (int cc = 0; cc < 8; ++cc) {
            int64_t v;
            float wc;
            if (!emc_voxel::trilinear_corner(u, g.side, cc, &v, &wc) || wc == 0.0f) continue;
            red_add_v2(g.acc + v, wc * val, wc * wT);
          }
        }
      }
    }
  }
};

// Kg[slot][j] = Kh[pattern of slot][j] (FP16 counts, rows of Ppad; zero rows
// for the padding slots), 16-byte copies.
__global__ void gather_rows_kernel(const __half* Kh, int64_t Ppad, const int32_t* slot_pat,
                                   int64_t S, __half* Kg) {
  const int64_t s = blockIdx.x;  // one block per slot
  if (s >= S) return;
  const int p = slot_pat[s];
  const int64_t n16 = Ppad / 8;
  const uint4* src = reinterpret_cast<const uint4*>(Kh + (int64_t)(p < 0 ? 0 : p) * Ppad);
  uint4* dst = reinterpret_cast<uint4*>(Kg + s * Ppad);
  for (int64_t i = threadIdx.x; i < n16; i += blockDim.x)
    dst[i] = p < 0 ? make_uint4(0, 0, 0, 0) : src[i];
}

// The same rows built from the counts' photon lists (kptr [N+1], kidx =
// active pixel, kval = count): the row is zeroed in shared memory, the
// pattern's photons scattered into it as FP16 (exact: integers <= 2048), and
// written out whole, so only the rows are written and only the photon lists
// read (the dense gather reads every row of Kh as well).
__global__ void slot_rows_kernel(const int64_t* kptr, const int32_t* kidx, const float* kval,
                                 int64_t Ppad, const int32_t* slot_pat, int64_t S, __half* Kg) {
  extern __shared__ uint4 srow[];  // [Ppad / 8]
  const int64_t s = blockIdx.x;  // one block per slot
  if (s >= S) return;
  const int p = slot_pat[s];
  const int64_t n16 = Ppad / 8;
  for (int64_t i = threadIdx.x; i < n16; i += blockDim.x) srow[i] = make_uint4(0, 0, 0, 0);
  __syncthreads();
  if (p >= 0) {
    __half* h = reinterpret_cast<__half*>(srow);
    for (int64_t t = kptr[p] + threadIdx.x; t < kptr[p + 1]; t += blockDim.x)
      h[kidx[t]] = __float2half_rn(kval[t]);
  }
  __syncthreads();
  uint4* dst = reinterpret_cast<uint4*>(Kg + s * Ppad);
  for (int64_t i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = srow[i];
}

// The grouped compress operand: A[r][q] = P / (T_r phi) of rotation r and the
// q-th slot of its cell as FP16 hi + lo, zero from the cell's slot count up to
// the next multiple of 64 (the contraction's k-blocks), and zero rows for
// rotations with T_r <= 1e-10.  One block per rotation.
__global__ void p_split_kernel(const GroupArgs g, const int32_t* cell_of, const float* T,
                               int64_t ldA, __half* Ahi, __half* Alo) {
  const int64_t r = blockIdx.x;
  const int c = cell_of[r];
  const int32_t gc = g.gcnt[c];
  if (gc == 0) return;
  const int64_t k = r - g.mbeg[c];
  const float Tr = T[r];
  const float inv = Tr > 1e-10f ? 1.0f / Tr : 0.0f;
  const int32_t width = (gc + 63) / 64 * 64;
  const float* src = g.Pt + g.goff[c] + k * gc;
  for (int32_t q = threadIdx.x; q < width; q += blockDim.x) {
    const float v = q < gc ? src[q] * inv : 0.0f;
    const __half hi = __float2half_rn(v);
    Ahi[r * ldA + q] = hi;
    Alo[r * ldA + q] = __float2half_rn(v - __half2float(hi));
  }
}

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
  const dim3 grid((unsigned)((a.N + 31) / 32), (unsigned)((a.n_cells + kCellWarps - 1) / kCellWarps));
  targets_kernel<<<grid, 32 * kCellWarps, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_scatter_targets(const int32_t* cand, const float* cmass, int64_t N, int m,
                                  int n_cells, float* t, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(t, 0, sizeof(float) * N * n_cells, st);
  if (e != cudaSuccess) return e;
  scatter_targets_kernel<<<(unsigned)((N * m + 255) / 256), 256, 0, st>>>(cand, cmass, N, m, n_cells, t);
  return cudaGetLastError();
}

__global__ void fill_f32_kernel(float* x, int64_t n, float v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = v;
}

cudaError_t launch_log_targets(const TargetArgs& a, cudaStream_t st) {
  const dim3 grid((unsigned)((a.N + 31) / 32), (unsigned)((a.n_cells + kCellWarps - 1) / kCellWarps));
  log_targets_kernel<<<grid, 32 * kCellWarps, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_scatter_log_targets(const int32_t* cand, const float* lcmass, int64_t N, int m,
                                      int n_cells, float* t, cudaStream_t st) {
  const int64_t n = N * n_cells;
  fill_f32_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(t, n,
                                                                                     -INFINITY);
  scatter_targets_kernel<<<(unsigned)((N * m + 255) / 256), 256, 0, st>>>(cand, lcmass, N, m,
                                                                          n_cells, t);
  return cudaGetLastError();
}

cudaError_t launch_select_topk(const float* probs, const float* log_keep, const int32_t* mcnt,
                               int64_t N, int C, int top_k, int m, float mass_target,
                               float keep_tail, int32_t* cand, float* mass, cudaStream_t st) {
  select_topk_kernel<<<(unsigned)((N + 7) / 8), 256, 0, st>>>(probs, log_keep, mcnt, N, C, top_k,
                                                              m, mass_target, keep_tail, cand,
                                                              mass);
  return cudaGetLastError();
}

cudaError_t launch_audit(const AuditArgs& a, int64_t n_audit, cudaStream_t st) {
  if (n_audit <= 0) return cudaSuccess;
  audit_kernel<<<(unsigned)n_audit, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_group_list_count(const GroupArgs& g, float theta, int64_t* cnt,
                                    cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(int64_t) * g.R, st);
  if (e != cudaSuccess) return e;
  group_list_kernel<0><<<(unsigned)((g.N + 7) / 8), 256, 0, st>>>(
      g, theta, reinterpret_cast<unsigned long long*>(cnt), nullptr, nullptr, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_group_list_fill(const GroupArgs& g, float theta, int64_t* cursor,
                                   const int64_t* rowoff, int32_t* pat, float* xv,
                                   cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(int64_t) * g.R, st);
  if (e != cudaSuccess) return e;
  group_list_kernel<1><<<(unsigned)((g.N + 7) / 8), 256, 0, st>>>(
      g, theta, reinterpret_cast<unsigned long long*>(cursor), rowoff, pat, xv);
  return cudaGetLastError();
}

cudaError_t launch_proposed_resp(const GroupArgs& g, float* P, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(P, 0, sizeof(float) * g.N * g.R, st);
  if (e != cudaSuccess) return e;
  proposed_resp_kernel<<<(unsigned)((g.N + 7) / 8), 256, 0, st>>>(g, P);
  return cudaGetLastError();
}

cudaError_t launch_select(const float* probs, const float* keep, int64_t N, int C, int min_m,
                          int m, float mass_target, float keep_mass, int32_t* cand, float* mass,
                          cudaStream_t st) {
  select_kernel<<<(unsigned)((N + 7) / 8), 256, 0, st>>>(probs, keep, N, C, min_m, m, mass_target,
                                                         keep_mass, cand, mass);
  return cudaGetLastError();
}

cudaError_t launch_group_maximize(const GroupArgs& g, int64_t n_mtiles, cudaStream_t st) {
  if (n_mtiles > 0) {
    OpGroupLL op{g};
    tile_kernel<<<(unsigned)n_mtiles, kTileThreads, 0, st>>>(op);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  group_softmax_kernel<<<(unsigned)((g.N + 7) / 8), 256, 0, st>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_group_softmax(const GroupArgs& g, cudaStream_t st) {
  group_softmax_kernel<<<(unsigned)((g.N + 7) / 8), 256, 0, st>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_gather_slots(const __half* Kh, int64_t Ppad, const int32_t* slot_pat, int64_t S,
                                __half* Kg, cudaStream_t st) {
  if (S == 0) return cudaSuccess;
  gather_rows_kernel<<<(unsigned)S, 256, 0, st>>>(Kh, Ppad, slot_pat, S, Kg);
  return cudaGetLastError();
}

bool slot_rows_fit(int64_t Ppad) { return Ppad * 2 <= 200 * 1024; }

cudaError_t launch_slot_rows(const int64_t* kptr, const int32_t* kidx, const float* kval,
                             int64_t Ppad, const int32_t* slot_pat, int64_t S, __half* Kg,
                             cudaStream_t st) {
  const size_t smem = (size_t)Ppad * sizeof(__half);
  cudaError_t e = cudaFuncSetAttribute(slot_rows_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (S > 0) slot_rows_kernel<<<(unsigned)S, 256, smem, st>>>(kptr, kidx, kval, Ppad, slot_pat, S, Kg);
  return cudaGetLastError();
}

cudaError_t launch_p_split(const GroupArgs& g, const int32_t* cell_of, int64_t R, const float* T,
                           int64_t ldA, __half* Ahi, __half* Alo, cudaStream_t st) {
  p_split_kernel<<<(unsigned)R, 128, 0, st>>>(g, cell_of, T, ldA, Ahi, Alo);
  return cudaGetLastError();
}

cudaError_t launch_group_compress(const GroupArgs& g, int64_t n_ctiles, cudaStream_t st) {
  if (n_ctiles == 0) return cudaSuccess;
  OpGroupCmp op{g};
  dim3 grid((unsigned)n_ctiles, (unsigned)((g.npa + TN - 1) / TN));
  tile_kernel<<<grid, kTileThreads, 0, st>>>(op);
  return cudaGetLastError();
}

}  // namespace emc
