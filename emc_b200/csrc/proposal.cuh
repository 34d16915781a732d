// Learned rotation proposal: launch interface (kernels in proposal.cu).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace emc {

// x[p][S*S] = log(1 + sum of the counts of each 2x2 pixel block), S = side/2.
cudaError_t launch_features(const float* K, const int32_t* pix, int64_t N, int64_t npa, int side,
                            int S, float* x, cudaStream_t st);

// t[p][c] = sum of the responsibilities of cell c's fine rotations.
struct TargetArgs {
  int64_t N, R;
  int n_cells;
  const int32_t* cell;     // [R] cell of every fine rotation
  const int64_t* mbeg;     // [n_cells] first rotation of each cell (rotations sorted by cell)
  const int32_t* mcnt;     // [n_cells] its rotation count
  const float* P;          // FP32 responsibilities [R][ldP] (FP32 path) or nullptr
  const double* L64;       // log targets of FP32 contexts: the FP64 log-likelihood [R][ldP]
  int64_t ldP;
  const float* Y;          // otherwise from the mixed path's Y and lse
  int64_t ldY;
  int poisson;
  const double* lse;
  const float* scaling;    // phi used for LL (gaussian)
  const double* rowstat;
  const double* patstat;
  double gauss_inv;
  float* t;                // [N][n_cells]
};
cudaError_t launch_targets(const TargetArgs& a, cudaStream_t st);
// The same after a proposed iteration: t[p][cand[p][i]] = cmass[p][i], 0 elsewhere.
cudaError_t launch_scatter_targets(const int32_t* cand, const float* cmass, int64_t N, int m,
                                   int n_cells, float* t, cudaStream_t st);

// cand[p][0..m): with keep (optional, [N][C]) first the most probable cells
// of keep[p] that have keep > 0, until at least min_m are taken and their keep
// total reaches keep_mass; then the most probable remaining cells of probs[p]
// in order until at least min_m are taken and their probs total reaches
// mass_target, at most m (the rest -1); mass[p] = that total.
cudaError_t launch_select(const float* probs, const float* keep, int64_t N, int C, int min_m,
                          int m, float mass_target, float keep_mass, int32_t* cand, float* mass,
                          cudaStream_t st);

// Pairs (pattern, selected cell) grouped by cell: group c holds pairs
// gbeg[c] .. gbeg[c]+gcnt[c]-1, pair q belongs to pattern gpair[q]; pattern
// p's i-th selected cell is cand[p*m+i] (-1: none, and none after it) and
// its pair is ppos[p*m+i].  Cell c's
// fine rotations are mbeg[c] .. mbeg[c]+mcnt[c]-1.
struct GroupArgs {
  int64_t N, npa, MM;      // MM: row stride of Y (>= largest cell)
  int64_t R;               // fine rotations (responsibility export)
  int n_cells, m, poisson;
  const int64_t* mbeg;
  const int32_t* mcnt;
  const int64_t* gbeg;
  const int32_t* gcnt;
  const int32_t* gpair;
  const int64_t* ppos;
  const int32_t* cand;
  const int64_t* goff;     // offset of cell c's [mcnt][gcnt] block in Pt
  const float* S;          // FP32 slice operand [R][ldS] (log W or S), or nullptr ->
  const __half* hi;        // FP16 hi + lo [Rpad][ldS]
  const __half* lo;
  int64_t ldS;
  const float* K;          // [N][npa]
  const float* scaling;    // phi used for LL
  const double* rowstat;   // poisson: sum W_r; gaussian: sum S_r^2
  const double* patstat;   // sum K^2
  const double* patsum;    // sum K
  double gauss_inv;
  float* Y;                // [pairs][MM]
  float* Pt;               // per cell [mcnt][gcnt]: P / phi_new (nullptr: not needed)
  float* T;                // [R] (zeroed by the caller)
  double* lse;             // [N]
  double* plogp;           // [N]
  float* new_scaling;      // [N]
  float* cmass;            // [N][m] responsibility mass of each candidate cell
  float* lcmass;           // optional [N][m]: its natural log in FP64 (-inf when 0)
  int32_t* best_rot;       // [N] most probable rotation among the candidates
  float* best_p;           // [N] its responsibility
  // tile lists: mtiles (cell, member offset, pair offset) of the grouped
  // maximize; ctiles (cell, member offset) of the grouped compress
  const int4* mtiles;
  const int4* ctiles;
  // insertion (compress epilogue) into interleaved (model, weight) accumulators
  const float* rotw;       // [R]
  const float* quat;       // [R][4]
  const float *cx, *cy, *cz;
  const int32_t* ins;      // [npa] insertion mask (== 1)
  int side, interp;
  float2* acc;             // [M] zeroed by the caller
};
cudaError_t launch_group_maximize(const GroupArgs& g, int64_t n_mtiles, cudaStream_t st);
// The per-pattern softmax of the grouped maximize alone (after the tcgen05 contraction).
cudaError_t launch_group_softmax(const GroupArgs& g, cudaStream_t st);
// Gathered FP16 counts of the tcgen05 grouped contractions (A of the
// maximize, MN-major B of the compress): Kg[slot][Ppad] from Kh[Npad][Ppad];
// slot_pat[slot] = pattern, -1 for padding (zero).
cudaError_t launch_gather_slots(const __half* Kh, int64_t Ppad, const int32_t* slot_pat, int64_t S,
                                __half* Kg, cudaStream_t st);
// The same rows from the counts' photon lists (kptr [N+1], kidx, kval), each
// row built in shared memory: Ppad FP16 must fit (slot_rows_fit).
bool slot_rows_fit(int64_t Ppad);
cudaError_t launch_slot_rows(const int64_t* kptr, const int32_t* kidx, const float* kval,
                             int64_t Ppad, const int32_t* slot_pat, int64_t S, __half* Kg,
                             cudaStream_t st);
// A[r][q] = P / (T_r phi) of the grouped compress as FP16 hi + lo ([R][ldA]).
cudaError_t launch_p_split(const GroupArgs& g, const int32_t* cell_of, int64_t R, const float* T,
                           int64_t ldA, __half* Ahi, __half* Alo, cudaStream_t st);
cudaError_t launch_group_compress(const GroupArgs& g, int64_t n_ctiles, cudaStream_t st);

// lt[p][c] = natural log of cell c's responsibility mass, summed in FP64
// (-inf when it is 0); t of TargetArgs receives it.
cudaError_t launch_log_targets(const TargetArgs& a, cudaStream_t st);
// The same after a proposed iteration from the candidates' log masses
// (-inf outside the candidate cells).
cudaError_t launch_scatter_log_targets(const int32_t* cand, const float* lcmass, int64_t N, int m,
                                      int n_cells, float* t, cudaStream_t st);
// Top-k selection: cells in order of log_keep (finite values) until they hold
// at least top_k fine rotations and (keep_tail > 0) all but keep_tail of the
// previous posterior, then cells in order of probs until the probs total
// reaches mass_target; at most m; either input may be null.
cudaError_t launch_select_topk(const float* probs, const float* log_keep, const int32_t* mcnt,
                               int64_t N, int C, int top_k, int m, float mass_target,
                               float keep_tail, int32_t* cand, float* mass, cudaStream_t st);

// Dense audit of sampled patterns (see audit_kernel): captured[a] = share of
// audited pattern pat[a]'s responsibility on the fine rotations of its
// candidate cells (cand [N][m]), from LL64 [R][ld] or Y [R][ld].
struct AuditArgs {
  int64_t R, ld;
  int m, poisson;
  const int64_t* pat;      // [n_audit] global pattern index
  const int32_t* cand;     // [N][m]
  const int32_t* cell;     // [R]
  const double* LL64;      // FP32 contexts: log-likelihood, or nullptr ->
  const float* Y;          // mixed: Y of the audit contraction
  const float* scaling;    // [n_audit] phi used for LL (gaussian)
  const double* rowstat;   // [R]
  const double* patstat;   // [n_audit] gaussian: sum K^2
  double gauss_inv;
  float* captured;         // [n_audit]
};
cudaError_t launch_audit(const AuditArgs& a, int64_t n_audit, cudaStream_t st);
// Responsibility lists of a proposed iteration (after the grouped softmax):
// count[r] of the patterns with P >= theta T_r, then the entries
// (pattern, value) at rowoff[r] (cursor [R] scratch); for launch_list_compress.
cudaError_t launch_group_list_count(const GroupArgs& g, float theta, int64_t* cnt,
                                    cudaStream_t st);
cudaError_t launch_group_list_fill(const GroupArgs& g, float theta, int64_t* cursor,
                                   const int64_t* rowoff, int32_t* pat, float* xv,
                                   cudaStream_t st);
// FP32 responsibilities [R][N] of the last proposed iteration (zero outside
// each pattern's candidate cells).
cudaError_t launch_proposed_resp(const GroupArgs& g, float* P, cudaStream_t st);

}  // namespace emc
