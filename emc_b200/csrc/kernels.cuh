// Launchers of the engine's CUDA kernels (all asynchronous on `st`).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace emc {

enum ExpandOut { EXP_F32 = 0, EXP_LOG_F32 = 1, EXP_F16_SPLIT = 2 };
enum StatKind { STAT_NONE = 0, STAT_SUMSQ = 1, STAT_SUM = 2 };

struct ExpandArgs {
  const float* model;   // side^3
  const float* quat;    // [R][4]
  const float* cx;      // [npix] pixel coordinates (compact or full grid)
  const float* cy;
  const float* cz;
  const int32_t* stat_mask;  // pixels counted in the row statistic (nullptr: all)
  int64_t R, npix, ld;  // ld: output row stride in elements (>= npix; extra columns zeroed)
  int side, interp;
  int out;              // ExpandOut
  int stat;             // StatKind (statistic of the slice value W, before any log)
  float floor_;         // log floor for EXP_LOG_F32 / log mode of EXP_F16_SPLIT
  int log_split;        // EXP_F16_SPLIT: split log(max(W,floor)) instead of W
  float* out_f32;
  __half* out_hi;
  __half* out_lo;
  double* rowstat;      // [R] or nullptr
  // optional, nearest + EXP_F16_SPLIT: per-voxel table from launch_expand_table
  // ([side^3 + 1], the last entry for pixels that fall outside the grid)
  const uint2* tab;
  // optional, trilinear: the stencil table of launch_tri_table
  const float4* tri;
};
cudaError_t launch_expand(const ExpandArgs& a, cudaStream_t st);
// Trilinear stencil table: per base voxel of [-1, side)^3 the model at its 8
// corners (0 outside the grid), tri_table_entries(side) float4.
int64_t tri_table_entries(int side);
cudaError_t launch_tri_table(const float* model, int side, float4* tri, cudaStream_t st);
// tab[v] = (bits of model[v], FP16 hi | lo << 16 of the split operand value:
// log(max(model[v], floor)) when log_split, else model[v]) for v < M, and
// tab[M] the same for a pixel outside the grid (value 0).
cudaError_t launch_expand_table(const float* model, int64_t M, float floor_, int log_split,
                                uint2* tab, cudaStream_t st);

// LL[r][p] (ld = ldLL) from slices A[R][ldA] and counts K[N][ldK] over npa
// active pixels (pix: optional column indirection into A and K).
struct LLArgs {
  const float* A;
  const float* K;
  const int32_t* pix;
  const float* scaling;  // [N]
  const double* rowstat; // poisson: sum_j W_rj
  int64_t R, N, npa, ldA, ldK, ldLL;
  double gauss_inv;      // 1 / (2 cnt sigma^2)
  int poisson;
  float* LL;
  double* LL64;          // when set, LL is written here in FP64 instead (LL unused)
};
cudaError_t launch_ll_fp32(const LLArgs& a, cudaStream_t st);

// Photon-list form of the poisson log-likelihood (FP32 path):
// LL[r][p] = sum over the non-zero pixels e of pattern p of K_e log W[r][j_e]
//            - phi_p sum W_r,
// from the counts in CSR (row_ptr [N+1], col = compact pixel, val = count)
// and log W pixel-major (logWT [npa][ldT], ldT >= R).
struct SparseLLArgs {
  const int64_t* row_ptr;
  const int32_t* col;
  const float* val;
  const float* logWT;
  int64_t ldT;
  const float* scaling;
  const double* rowstat;  // sum W_r
  int64_t R, N;
  float* LL;              // [R][N]
  double* LL64;           // when set, [R][N] in FP64 instead of LL
};
// ldT % 4 == 0 and logWT 16-byte aligned (each thread gathers 4 rotations).
cudaError_t launch_ll_sparse(const SparseLLArgs& a, cudaStream_t st);
// Slice sums from the counts in CSC (col_ptr [npa+1] over active pixels, row
// = pattern, val = K / phi of that pattern) and the responsibilities
// pattern-major (PT [N][ldT], ldT >= R, % 4 == 0):
//   U[r][j] = (sum over the pixel's entries val * PT[p][r]) / T_r   (T_r > 1e-30)
struct SparseCmpArgs {
  const int64_t* col_ptr;
  const int32_t* row;
  const float* val;
  const float* PT;
  int64_t ldT;
  const float* T;
  int64_t R, npa;
  float* U;               // [R][npa]
};
cudaError_t launch_compress_sparse(const SparseCmpArgs& a, cudaStream_t st);
// val_out[e] = val[e] / scaling[row[e]] over nnz entries.
cudaError_t launch_scale_entries(const float* val, const int32_t* row, const float* scaling,
                                 int64_t nnz, float* val_out, cudaStream_t st);
// logWT[j][r] = S[r][j] (tiled transpose, [R][npa] -> [npa][ldT]).
cudaError_t launch_transpose(const float* S, int64_t R, int64_t npa, float* ST, int64_t ldT,
                             cudaStream_t st);
// CSR of the non-zero entries of K [N][npa]: nnz per row (pass 1), then the
// entries in pixel order (pass 2, row_ptr given).
cudaError_t launch_csr_count(const float* K, int64_t N, int64_t npa, int64_t* count,
                             cudaStream_t st);
cudaError_t launch_csr_fill(const float* K, int64_t N, int64_t npa, const int64_t* row_ptr,
                            int32_t* col, float* val, cudaStream_t st);

// Per-pattern softmax over r of X[r][p] (in place), FP32 arithmetic as the
// reference; plogp_part[blockIdx] receives sum P log P partials (FP64) and
// lse[p] (optional) the pattern's log-sum-exp.
// The same per-pattern softmax from an FP64 log-likelihood L [R][N] into the
// FP32 responsibilities P [R][N].
cudaError_t launch_softmax_from_f64(const double* L, float* P, int64_t R, int64_t N,
                                    double* plogp_part, int* nparts, double* lse,
                                    cudaStream_t st);
cudaError_t launch_softmax_fp32(float* X, int64_t R, int64_t N, double* plogp_part,
                                int* nparts, double* lse, cudaStream_t st);
// sum of x log x over n floats into *out (FP64).
cudaError_t launch_xlogx_sum(const float* x, int64_t n, double* out, double* scratch,
                             cudaStream_t st);

// den_part[rt][p] = sum_{r in tile rt} P_rp sum_j S_rj K_pj (gaussian scaling).
struct CrossArgs {
  const float* S;
  const float* K;
  const int32_t* pix;
  const float* P;        // [R][N]
  int64_t R, N, npa, ldS, ldK;
  double* den_part;      // [ceil(R/128)][N]
};
cudaError_t launch_scaling_cross(const CrossArgs& a, cudaStream_t st);
// den[p] = sum_r P_rp w_r   (poisson scaling), deterministic two-level reduce.
cudaError_t launch_scaling_rowweighted(const float* P, const double* w, int64_t R, int64_t N,
                                       double* den_part, int64_t* nparts, cudaStream_t st);
// phi_p = num_p / sum_k den_part[k][p] where both are positive, else unchanged.
cudaError_t launch_scaling_finish(const double* num, const double* den_part, int64_t nparts,
                                  int64_t N, float* scaling, cudaStream_t st);
// num[p] = sum_j K_pj^2 (gauss) or sum_j K_pj (poisson) over active pixels.
cudaError_t launch_pattern_stats(const float* K, const int32_t* pix, int64_t N, int64_t npa,
                                 int64_t ldK, int squares, double* num, cudaStream_t st);

// T[r] = sum_p P[r][p].
cudaError_t launch_row_sums(const float* P, int64_t R, int64_t N, float* T, cudaStream_t st);
// best[p] = argmax_r P[r][p], bestv[p] = its value.
cudaError_t launch_col_argmax(const float* P, int64_t R, int64_t N, int32_t* best, float* bestv,
                              cudaStream_t st);

// U[r][pix j] = sum_p P_rp K_pj / phi_p, divided by T_r where T_r > 1e-10.
struct CompressArgs {
  const float* P;
  const float* K;
  const int32_t* pix;    // optional: column j of U and K is pix[j]
  const float* scaling;
  const float* T;
  int64_t R, N, npa, ldK, ldU;
  float* U;
};
cudaError_t launch_compress_fp32(const CompressArgs& a, cudaStream_t st);

// model[v] += w_r U_rj / T_r ... insertion of the averaged slices
// (U already divided by T): model += rotw_r T_r U_rj, weight += rotw_r T_r.
struct InsertArgs {
  const float* U;        // [R][ldU]
  const float* T;        // [R]
  const float* Tskip;    // [R] T_r over all pattern shards for the <= 1e-10 skip (nullptr: T)
  const float* rotw;     // [R]
  const float* quat;
  const float* cx;
  const float* cy;
  const float* cz;
  const int32_t* ins;    // per pixel: insert when == 1
  int64_t R, npix, ldU;
  int side, interp;
  float* model;
  float* weight;
  // deterministic insertion: fixed-point limbs [M][8] (fixed.cuh) instead of
  // FP32 atomics into model and weight
  unsigned long long* acc64;
};
cudaError_t launch_insert(const InsertArgs& a, cudaStream_t st);
// The fixed-point sums (fixed.cuh) as FP32 pairs a[i stride], b[i stride].
cudaError_t launch_fixed_to_pairs(const unsigned long long* acc64, int64_t M, float* a, float* b,
                                  int64_t stride, cudaStream_t st);

// model = weight > 0 ? model / weight : 0; then model /= mean; stats[0] = mean,
// stats[1] = max after normalisation.  fp64 selects the FP64 division.
cudaError_t launch_normalize_model(float* model, const float* weight, int64_t M, int fp64,
                                   double* scratch, double* stats, cudaStream_t st);
// Same from interleaved (model, weight) accumulators; writes model and weight.
cudaError_t launch_normalize_acc(const float2* acc, float* model, float* weight, int64_t M,
                                 double* scratch, double* stats, cudaStream_t st);
cudaError_t launch_model_max(const float* model, int64_t M, double* scratch, double* out,
                             cudaStream_t st);
cudaError_t launch_fill(float* x, int64_t n, float v, cudaStream_t st);
cudaError_t launch_sum_f64(const double* x, int64_t n, double* out, cudaStream_t st);
// bad[0] += number of entries of x that are negative, NaN or infinite.
cudaError_t launch_count_invalid(const float* x, int64_t n, int* bad, cudaStream_t st);

}  // namespace emc
