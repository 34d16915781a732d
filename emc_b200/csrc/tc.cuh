// Mixed-precision (tcgen05) path: launch interface.
#pragma once
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace emc {

// Device-side status of the tensor-core kernels: code != 0 when a bounded
// wait gave up (the kernel then drained its copies, freed TMEM and returned).
struct TcStatus {
  int code;
  int where;
  int block;
  int pad;
};
enum { TC_OK = 0, TC_TIMEOUT = 1 };

// K-step (FP16 elements per shared-memory row) of the two contractions; the
// tensor maps of their operands use it as the inner box size.
constexpr int kMaximizeBK = 32;
constexpr int kCompressBK = 64;

bool tc_encode_2d(CUtensorMap* tm, const void* base, uint64_t inner, uint64_t rows,
                  uint32_t box_rows, uint32_t box_inner);
// One bounded wait that cannot succeed, given up after limit_ns: records
// TC_TIMEOUT (site 90) in *status the way the contractions do.
cudaError_t launch_wait_probe(TcStatus* status, uint64_t limit_ns, cudaStream_t st);
// The same for a matrix whose rows are ld >= inner elements apart (reads past
// `inner` are zero-filled).
bool tc_encode_2d_strided(CUtensorMap* tm, const void* base, uint64_t inner, uint64_t rows,
                          uint64_t ld, uint32_t box_rows, uint32_t box_inner);

// Maximize contraction: acc[p][r] = sum_j K[p][j] (B_hi[r][j] + B_lo[r][j]),
// 128 patterns x 256 rotations per tile.  Epilogue writes Y[r][p] (LL for
// poisson, the cross term C for gaussian) and per pattern and rotation tile
// the online log-sum-exp partials (m, s, d, q) described in kernels_tc.cu.
struct MaxEpiArgs {
  int64_t N, R, ldY;
  int poisson;
  const float* scaling;    // [N] current phi
  const double* rowstat;   // [R] poisson: sum W_r; gaussian: sum S_r^2
  const double* patstat;   // [N] gaussian: sum K_p^2
  double gauss_inv;        // 1 / (2 cnt sigma^2)
  float* Y;                // [R][ldY]
  float4* part;            // [Rpad/256][N]
};
// raster: rotation tiles per band of the tile order (see kernels_tc.cu).
cudaError_t launch_maximize_tc(const CUtensorMap& tmK, const CUtensorMap& tmBhi,
                               const CUtensorMap& tmBlo, int64_t Mpad, int64_t Rpad,
                               int64_t Kpad, const MaxEpiArgs& e, TcStatus* status,
                               int num_sms, cudaStream_t st, int raster);

// The same contraction on SM pairs (cta_group::2): 256 patterns x 256
// rotations per pair, 64-wide K-steps; the tensor maps have boxes of 128 rows
// x 64 (kPairBoxK) for the counts and for each half of the slice operand.
constexpr int kPairBoxK = 64;
cudaError_t launch_maximize_pair_tc(const CUtensorMap& tmK, const CUtensorMap& tmBhi,
                                    const CUtensorMap& tmBlo, int64_t Mpad, int64_t Rpad,
                                    int64_t Kpad, const MaxEpiArgs& e, TcStatus* status,
                                    int num_sms, cudaStream_t st, int raster);

// Compress contraction: acc[r][j] = sum_p (P'_hi + P'_lo)[r][p] Kt[j][p] with
// P' = c0 P / (T_r phi_p), i.e. the averaged slice U_r / T_r; 128 rotations x
// 256 pixels per tile, inserted in the epilogue.
struct CmpEpiArgs {
  int64_t R, npa;
  int side, interp;
  float inv_c0;            // undo the global scale of P'
  const float* quat;       // [R][4]
  const float* rotw;       // [R]
  const float* T;          // [R]
  const float* Tskip;      // [R] T_r over all pattern shards for the <= 1e-10 skip
  const float* cx;         // [npa] active-pixel coordinates
  const float* cy;
  const float* cz;
  const int32_t* ins;      // [npa] insert flag (mask == 1)
  float2* acc;             // [side^3] interleaved (model, weight) accumulators
  unsigned long long* acc64;  // or, when set, fixed-point limbs [side^3][8] (fixed.cuh)
  // optional: the launch returns at once unless *gate_count > gate_cap (the
  // dense form as the fallback of responsibility lists that overflowed)
  const unsigned long long* gate_count;
  int64_t gate_cap;
};
// raster: rotation tiles per band of the tile order.
cudaError_t launch_compress_tc(const CUtensorMap& tmPhi, const CUtensorMap& tmPlo,
                               const CUtensorMap& tmKt, int64_t Rpad, int64_t Ppad,
                               int64_t Npad, const CmpEpiArgs& e, TcStatus* status, int num_sms,
                               cudaStream_t st, int raster);

// The compress contraction on SM pairs: 256 rotations x 256 pixels per
// pair, 64-wide K-steps; Kt's tensor map has boxes of 128 rows x 64.
cudaError_t launch_compress_pair_tc(const CUtensorMap& tmPhi, const CUtensorMap& tmPlo,
                                    const CUtensorMap& tmKt, int64_t Rpad, int64_t Ppad,
                                    int64_t Npad, const CmpEpiArgs& e, TcStatus* status,
                                    int num_sms, cudaStream_t st, int raster);

// Tile of a grouped contraction (learned proposal): TMA origins of the two
// operands (row, k offset), its k-block count, and the group (cell) with the
// tile's first row inside the group.
struct TileDesc {
  int32_t a_row, a_k0, b_row, b_k0;
  int32_t k_blocks, cell, local0, set;  // set: tensor maps / epilogue of the tile's dataset
};

// The four operand tensor maps of a contraction (A, A's hi/lo partner, B,
// B's partner), NSET sets for launches over several datasets.
template <int NSET>
struct TmapSet {
  CUtensorMap a0[NSET], a1[NSET], b0[NSET], b1[NSET];
};

// Grouped maximize: acc[slot][member] = sum_j Kg[slot][j] (B_hi + B_lo)[mbeg_c + member][j]
// over the selected cells; 128 slots x 256 members per tile (a cell has at
// most 256 members).  Writes Y[slot][member] (poisson LL, gaussian C).
struct GMaxEpiArgs {
  const TileDesc* tiles;
  const int32_t* mcnt;     // [n_cells] members per cell
  const int32_t* gcnt;     // [n_cells] slots (pairs) per cell
  const int32_t* gpair;    // [slots] pattern of each slot
  int poisson;
  const float* scaling;    // [N] phi used for LL
  const double* rowstat;   // [R] poisson: sum W_r
  float* Y;                // [slots][ldY]
  int64_t ldY;
};
cudaError_t launch_group_maximize_tc(const CUtensorMap& tmKg, const CUtensorMap& tmBhi,
                                     const CUtensorMap& tmBlo, int64_t n_tiles,
                                     const GMaxEpiArgs& e, TcStatus* status, int num_sms,
                                     cudaStream_t st);

// The same on SM pairs (cta_group::2): tiles of 256 slots (a_row and local0
// the pair tile's first slot) x 256 members, 64-wide K-steps; tensor maps with
// boxes of 128 rows x kPairBoxK (Kg, and each half of the slice operand).
cudaError_t launch_group_maximize_pair_tc(const CUtensorMap& tmKg, const CUtensorMap& tmBhi,
                                          const CUtensorMap& tmBlo, int64_t n_tiles,
                                          const GMaxEpiArgs& e, TcStatus* status, int num_sms,
                                          cudaStream_t st);

// Grouped compress: acc[member][j] = sum_q A[mbeg_c + member][q] Kg[slot0_c + q][j]
// with A = P / (T_r phi) as FP16 hi + lo (zero beyond the cell's slots);
// 128 members x 256 pixels per tile, inserted in the epilogue.  Kg is the B
// operand in its own [slot][pixel] layout (MN-major): its tensor map has
// boxes of 64 slot rows x 64 pixels; a tile's b_row is its first pixel and
// b_k0 its cell's first slot.
struct GCmpEpiArgs {
  const TileDesc* tiles;
  const int32_t* mcnt;
  int64_t npa;
  int side, interp;
  const float* quat;
  const float* rotw;
  const float* T;
  const float* cx;
  const float* cy;
  const float* cz;
  const int32_t* ins;
  float2* acc;
};
cudaError_t launch_group_compress_tc(const CUtensorMap& tmAhi, const CUtensorMap& tmAlo,
                                     const CUtensorMap& tmKg64, int64_t n_tiles,
                                     const GCmpEpiArgs& e, TcStatus* status, int num_sms,
                                     cudaStream_t st);

// Several datasets (contexts) in one persistent launch of each contraction:
// a tile list over all of them (set = dataset, local0 = row tile, cell =
// column tile) and each dataset's epilogue arguments.
constexpr int kMaxBatch = 8;
struct BatchMaxArgs {
  const TileDesc* tiles;
  const MaxEpiArgs* set;  // device array, one per dataset
};
struct BatchCmpArgs {
  const TileDesc* tiles;
  const CmpEpiArgs* set;  // device array, one per dataset
};
cudaError_t launch_batch_maximize_tc(const TmapSet<kMaxBatch>& maps, int64_t n_tiles,
                                     const BatchMaxArgs& e, TcStatus* status, int num_sms,
                                     cudaStream_t st);
// The same on SM pairs: tiles of 256 rows (local0 = pair row tile), tensor
// maps with boxes of 128 rows x kPairBoxK.
cudaError_t launch_batch_maximize_pair_tc(const TmapSet<kMaxBatch>& maps, int64_t n_tiles,
                                          const BatchMaxArgs& e, TcStatus* status, int num_sms,
                                          cudaStream_t st);
cudaError_t launch_batch_compress_pair_tc(const TmapSet<kMaxBatch>& maps, int64_t n_tiles,
                                          const BatchCmpArgs& e, TcStatus* status, int num_sms,
                                          cudaStream_t st);
cudaError_t launch_batch_compress_tc(const TmapSet<kMaxBatch>& maps, int64_t n_tiles,
                                     const BatchCmpArgs& e, TcStatus* status, int num_sms,
                                     cudaStream_t st);

// Responsibility pass of the mixed path: combine the tile partials per
// pattern (lse, new scaling, sum P log P), then two sweeps over Y: row sums
// T_r, and the compress operand P' = c0 P / (T_r phi_new) as FP16 hi + lo.
struct RespArgs {
  int64_t N, R, ldY, ldP, nparts;  // nparts = number of 256-rotation tiles
  int poisson;
  const float* Y;
  const float4* part;
  const float* scaling;    // phi used for LL
  const double* rowstat;
  const double* patstat;   // gaussian: sum K^2 (also the scaling numerator)
  const double* patsum;    // poisson: sum K (scaling numerator)
  double gauss_inv;
  double* lse;             // [N]
  double* plogp;           // [N] per-pattern sum P log P
  float* new_scaling;      // [N]
  float c0;                // global scale of P'
  __half* Phi;             // [Rpad][ldP]
  __half* Plo;
  float* Tpart;            // [ceil(N/1024)][R] partial sums of T_r
  float* T;                // [R]
  float* P32;              // optional [R][N] FP32 responsibilities
  // optional compaction during the row sums: every P_rp >= list_min is
  // appended as (r, p, P) at list_count[0]++ (capacity list_cap; entries past
  // it are counted, not written)
  unsigned long long* list_count;
  int64_t list_cap;
  int2* list_rp;
  float* list_P;
  float list_min;
  // rotation chunks: the sweep covers Y rows of rotations list_r0 .. list_r0
  // + R - 1 (R, rowstat and Y are the chunk's), appends (list_r0 + r, p, y)
  // with the stored y instead of P, and writes no Tpart (nullptr)
  int64_t list_r0;
  int list_store_y;
  // optional: write_kernel returns at once unless *gate_count > gate_cap
  const unsigned long long* gate_count;
  int64_t gate_cap;
};
cudaError_t launch_resp_pass(RespArgs& a, cudaStream_t st);
// The pass in two parts: combine + row sums (partials of T_r), then the
// FP16 compress operand (which also finishes T_r).
cudaError_t launch_resp_rowsums(RespArgs& a, cudaStream_t st);
cudaError_t launch_resp_write(RespArgs& a, cudaStream_t st);

// Responsibility lists (the compress operand as lists instead of P'):
// launch_resp_rowsums with RespArgs.list_* set compacts the entries, then
// launch_list_from_compact sorts them by rotation.
int64_t resp_list_blocks(int64_t N);
// rowoff[0..R] = exclusive prefix sums of rowtot (rowoff[R] = total).
cudaError_t launch_list_rowscan(const int64_t* rowtot, int64_t R, int64_t* rowoff,
                                cudaStream_t st);
// From the entries compacted by launch_resp_rowsums (n of them): T_r, then
// the lists sorted by rotation with x = P / (T_r phi_new), keeping entries
// with P >= rel_min T_r (rowtot, cursor: [R] scratch; rowoff [R+1]).  Order
// within a row is not fixed.  With n_dev the count is read on the device (n
// is then the capacity; a count above it leaves every list empty), so no host
// wait is needed, as in a captured graph.
cudaError_t launch_list_from_compact(RespArgs& a, int64_t n, float rel_min, int64_t* rowtot,
                                     int64_t* cursor, int64_t* rowoff, int32_t* pat, float* xv,
                                     cudaStream_t st,
                                     const unsigned long long* n_dev = nullptr);
// After a maximize over rotation chunks (launch_resp_rowsums per chunk with
// the running lse and list_store_y): P = exp(LL - lse_p) of the n candidates
// into Pv (their y stay in a.list_P), T_r = sum of P over each rotation's
// candidates (T64 [R] scratch; a.T), then the lists as launch_list_from_compact
// forms them from (a.list_rp, Pv).  a.R, a.rowstat: every rotation.
// Only the first step: Pv and the FP64 row sums T64 (atomics).
cudaError_t launch_cand_probs(const RespArgs& a, int64_t n, float* Pv, double* T64,
                              cudaStream_t st);
cudaError_t launch_list_from_candidates(RespArgs& a, int64_t n, float rel_min, float* Pv,
                                        double* T64, int64_t* rowtot, int64_t* cursor,
                                        int64_t* rowoff, int32_t* pat, float* xv, cudaStream_t st);
// Deterministic list order: the n entries (rp, v) sorted by (rotation,
// pattern) in place (stable radix sort; rp2, v2 [n] and hist
// [sort_hist_size(n)] scratch; N, R bound the fields) ...
int64_t sort_hist_size(int64_t n);
cudaError_t launch_sort_entries(int2* rp, float* v, int64_t n, int64_t N, int64_t R, int2* rp2,
                                float* v2, int64_t* hist, cudaStream_t st);
// ... T_r as the FP64 sum of each rotation's sorted entries in order
// (rowtot [R], rowoff [R+1] scratch) ...
cudaError_t launch_T_from_sorted(const int2* rp, const float* Pv, int64_t n, int64_t R,
                                 int64_t* rowtot, int64_t* rowoff, float* T, cudaStream_t st);
// ... and the lists of the entries with P >= rel_min T_r in sorted order,
// x = P / (T_r phi_new) (rowoff [R+1] of the lists; flag [2n + 2 +
// scan_scratch(n)] scratch).
int64_t scan_scratch(int64_t n);
cudaError_t launch_list_from_sorted(const int2* rp, const float* Pv, int64_t n, int64_t R,
                                    const float* T, const float* new_scaling, float rel_min,
                                    int64_t* rowtot, int64_t* rowoff, int64_t* flag,
                                    int32_t* pat, float* xv, cudaStream_t st);
// T_r from the row-sum partials (FP64, pattern-block order).
cudaError_t launch_finish_T(const float* Tpart, int64_t N, int64_t R, float* T, cudaStream_t st);

// Exports of a chunked iteration from its candidates (rp, Pv; n of them):
// dense P [R][N] (zeroed by the caller) ...
cudaError_t launch_cand_scatter(const int2* rp, const float* Pv, int64_t n, int64_t N, float* P,
                                cudaStream_t st);
// ... columns out[r][a] of patterns cols[a] (zeroed by the caller) ...
cudaError_t launch_cand_columns(const int2* rp, const float* Pv, int64_t n, const int64_t* cols,
                                int64_t ncols, float* out, cudaStream_t st);
// ... most probable rotation per pattern (largest LL from the stored y;
// ties to the lower rotation) and its P (key [N] scratch) ...
cudaError_t launch_cand_argmax(const RespArgs& a, int64_t n, unsigned long long* key,
                               int32_t* best, float* bestp, cudaStream_t st);
// ... and the responsibility mass per (pattern, cell) in FP64 (acc [N][C],
// zeroed by the caller), then t = acc or t = log(acc) (-inf where 0).
cudaError_t launch_cand_cells(const int2* rp, const float* Pv, int64_t n, const int32_t* cell,
                              int C, double* acc, cudaStream_t st);
cudaError_t launch_cells_out(const double* acc, int64_t count, int take_log, float* t,
                             cudaStream_t st);

// Compress from the lists with the counts' photon lists (kptr [N+1], kidx =
// active pixel, kval = count): one block per rotation accumulates its slice
// in shared memory (npa floats) and inserts it as the contraction's epilogue
// does (e.inv_c0 unused).
struct ListCmpArgs {
  const int64_t* rowoff;
  const int32_t* pat;
  const float* xv;
  const int64_t* kptr;
  const int32_t* kidx;
  const float* kval;
  CmpEpiArgs e;
  int ordered;  // sum each pixel's terms in list order (deterministic mode)
  // optional: the launch returns at once if *gate_count > gate_cap (lists
  // that overflowed their capacity are incomplete)
  const unsigned long long* gate_count;
  int64_t gate_cap;
};
cudaError_t launch_list_compress(const ListCmpArgs& a, cudaStream_t st);
// FP32 responsibilities [R][N] from Y and lse (readback / tests).
cudaError_t launch_resp_export(const RespArgs& a, float* P, cudaStream_t st);
// Most probable rotation of every pattern and its responsibility, from Y and lse.
cudaError_t launch_resp_argmax(const RespArgs& a, int32_t* best, float* bestp, cudaStream_t st);
// Builds the FP16 pattern operands: Kh[Npad][Ppad] and Kt[Ppad][Npad] from
// compact FP32 counts [N][npa]; bad[0] counts entries that are not integers in [0, 2048].
cudaError_t launch_pack_patterns(const float* K, int64_t N, int64_t npa, int64_t Npad,
                                 int64_t Ppad, __half* Kh, __half* Kt, int* bad,
                                 cudaStream_t st);

}  // namespace emc
