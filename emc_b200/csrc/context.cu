// Context API (include/emc_b200.h): one dataset resident in HBM, iterated
// in the order of the reference's main loop (emc.c:989-1084).
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/emc_b200.h"
#include "kernels.cuh"
#include "proposal.cuh"
#include "tc.cuh"
#include "tile.cuh"

namespace {
// An NVTX range over one stage of an iteration (nsys and ncu show the stages
// by name; without a profiler attached the calls do nothing), closed on every
// return path.
struct StageRange {
  explicit StageRange(const char* name) { nvtxRangePushA(name); }
  ~StageRange() { nvtxRangePop(); }
  StageRange(const StageRange&) = delete;
  StageRange& operator=(const StageRange&) = delete;
};
}  // namespace

using namespace emc;

namespace {

int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

__global__ void gather_cols_kernel(const float* src, int64_t rows, int64_t ld, const int32_t* pix,
                                   int64_t npa, float* dst) {
  const int64_t r = blockIdx.y;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < npa;
       j += (int64_t)gridDim.x * blockDim.x)
    dst[r * npa + j] = src[r * ld + pix[j]];
}

// Photon lists (CSR over patterns) into the compact counts: one warp per
// pattern; entries on masked-out pixels are dropped, entries outside the
// detector are counted in bad[0].  Counts are summed atomically (a pixel may
// appear once per photon); integer counts make the order irrelevant.
__global__ void scatter_photons_kernel(const int64_t* row_ptr, const int32_t* pix,
                                       const float* val, int64_t N, int64_t npix,
                                       const int32_t* compact_of, int64_t npa, float* K,
                                       int* bad) {
  const int64_t p = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= N) return;
  int nbad = 0;
  for (int64_t e = row_ptr[p] + lane; e < row_ptr[p + 1]; e += 32) {
    const int32_t i = pix[e];
    if (i < 0 || i >= npix) {
      ++nbad;
      continue;
    }
    const int32_t j = compact_of[i];
    if (j >= 0) atomicAdd(K + p * npa + j, val ? val[e] : 1.0f);
  }
  if (nbad) atomicAdd(bad, nbad);
}

__global__ void split_sum_kernel(const __half* hi, const __half* lo, int64_t R, int64_t ld,
                                 int64_t npa, const int32_t* rank, float* out) {
  const int64_t r = blockIdx.y;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < npa;
       j += (int64_t)gridDim.x * blockDim.x)
    out[r * npa + (rank ? rank[j] : j)] = __half2float(hi[r * ld + j]) + __half2float(lo[r * ld + j]);
}

// Responsibility columns of chosen patterns, out [R][n]:
//   dense FP32 path: P itself ([R][N]);
//   dense mixed path: exp(LL - lse) from Y (poisson LL, gaussian cross term);
//   proposed iteration: over each pattern's candidate cells (out zeroed).
__global__ void resp_cols_dense_kernel(const float* P, const float* Y, int64_t ld, int poisson,
                                       const float* scaling, const double* rowstat,
                                       const double* patstat, double gauss_inv, const double* lse,
                                       int64_t R, const int64_t* cols, int64_t n, float* out) {
  const int64_t total = R * n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / n, a = e - r * n, p = cols[a];
    if (P) {
      out[e] = P[r * ld + p];
      continue;
    }
    double ll = (double)Y[r * ld + p];
    if (!poisson) {
      const double phi = scaling[p];
      ll = (ll * 2.0 / phi - rowstat[r] - patstat[p] / (phi * phi)) * gauss_inv;
    }
    out[e] = (float)exp(ll - lse[p]);
  }
}

__global__ void resp_cols_proposed_kernel(const GroupArgs g, const int64_t* cols, int64_t n,
                                          float* out) {
  const int64_t a = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (a >= n) return;
  const int64_t p = cols[a];
  const double phi = g.scaling[p];
  const double c1 = 2.0 * g.gauss_inv / phi,
               c0 = g.poisson ? 0.0 : -g.patstat[p] / (phi * phi) * g.gauss_inv;
  for (int i = 0; i < g.m; ++i) {
    const int c = g.cand[p * g.m + i];
    if (c < 0) break;
    const int64_t q = g.ppos[p * g.m + i];
    for (int k = lane; k < g.mcnt[c]; k += 32) {
      const double y = (double)g.Y[q * g.MM + k];
      const double l = g.poisson ? y : fma(y, c1, c0 - g.rowstat[g.mbeg[c] + k] * g.gauss_inv);
      out[(g.mbeg[c] + k) * n + a] = (float)exp(l - g.lse[p]);
    }
  }
}

}  // namespace

// The compress lists keep the responsibilities P_rp >= kListRel T_r: a
// dropped entry moves its rotation's slice sum by less than 1e-12 (FP16 P'
// of the dense contraction rounds entries below 2^-25 of the row to zero).
// The row-sum sweep compacts P >= kListMinP first (rotations with T_r <=
// 1e-10 are not inserted, emc_atomic.cu:128, so nothing kept is below it).
constexpr float kListRel = 1e-12f;
constexpr float kListMinP = 1e-30f;
// Shared memory of the list compress: one FP32 per active pixel.
constexpr int64_t kListMaxPixels = 51200;
// A batched dataset keeps its own contraction launches when its maximize
// alone fills the persistent grid this many times over.
constexpr int64_t kAloneWaves = 8;

// Non-zero entries of a dense matrix as compressed rows (see build_rows).
struct SparseRows {
  int64_t* ptr = nullptr;   // [rows + 1]
  int32_t* idx = nullptr;   // column of each entry, ascending within a row
  float* val = nullptr;     // the entry
  float* aux = nullptr;     // optional second value per entry
  int64_t cap = 0, nnz = 0;
  bool valid = false;
};

struct emc_context {
  emc_config cfg{};
  std::string err;
  cudaStream_t st = nullptr;
  int num_sms = 148;
  int64_t N = 0, R = 0, npix = 0, M = 0, npa = 0;
  bool mixed = false, gauss = true;
  bool have_geom = false, have_rot = false, have_pat = false, have_model = false;
  int stage = 0;  // 0 ready to expand, 1 expanded, 2 maximized
  std::vector<void*> allocs;
  std::vector<size_t> alloc_bytes;  // size of each entry of allocs
  size_t mem_used = 0, mem_limit = 0;  // device bytes held; limit 0 = none

  // geometry (compact active pixels)
  int32_t* d_pix = nullptr;   // detector pixel of every compact (active) pixel
  int32_t* d_rank = nullptr;  // mixed: ascending position of every compact pixel
  int32_t* d_ins = nullptr;
  float *d_cx = nullptr, *d_cy = nullptr, *d_cz = nullptr;
  // rotations
  float *d_quat = nullptr, *d_rotw = nullptr;
  // patterns
  float* d_K = nullptr;      // [N][npa] FP32 counts on the active pixels
  float* d_stage = nullptr;  // [N][side^2] upload staging
  // photon-list upload staging (CSR) and the detector pixel -> compact map
  int64_t* d_sp_row = nullptr;
  int32_t* d_sp_pix = nullptr;
  float* d_sp_val = nullptr;
  int64_t sp_cap = 0;
  int32_t* d_compact_of = nullptr;
  double *d_patsq = nullptr, *d_patsum = nullptr;
  // model state
  float *d_model = nullptr, *d_weight = nullptr, *d_scaling = nullptr, *d_scaling_prev = nullptr;
  float* d_T = nullptr;
  float* d_Tskip = nullptr;  // T_r for the insertion skip: this context's T, or all shards' sum
  double* d_rowstat = nullptr;
  uint2* d_vtab = nullptr;  // mixed + nearest: per-voxel (W, split operand) table of the expand
  float4* d_tri = nullptr;  // trilinear: the expansion's stencil table (8 corners per base voxel)
  double* d_scratch = nullptr;  // reductions
  double* d_stats = nullptr;    // [0] mean [1] max [2] plogp [3] loglik
  // FP32 path
  float* d_S = nullptr;   // [R][npa]
  float* d_LL = nullptr;  // [R][N] responsibilities (FP32)
  double* d_LL64 = nullptr;  // [R][N] log-likelihood (FP64) the softmax reads
  double* d_den = nullptr;
  double* d_lse32 = nullptr;
  double* d_plogp_part = nullptr;
  // mixed path
  int64_t Npad = 0, Ppad = 0, Rpad = 0, nrt = 0;
  __half *d_Kh = nullptr, *d_Kt = nullptr, *d_Bhi = nullptr, *d_Blo = nullptr;
  __half *d_Phi = nullptr, *d_Plo = nullptr;
  float* d_Y = nullptr;
  // rotation chunks: Y holds y_rows rotations (R: one chunk); a chunked
  // maximize keeps its candidates (d_lcomp_rp / d_lcomp_P: rotation, pattern,
  // y) and their final P (d_cand_P) until the next maximize
  int64_t y_rows = 0, cand_n = 0, cand_cap_min = 0, cand_P_cap = 0;
  bool batched = false;  // a member of an emc_batch
  // deterministic insertion: fixed-point limbs [M][8] (fixed.cuh) and the
  // scratch of the (rotation, pattern) sort of the responsibility lists
  bool det = false;
  unsigned long long* d_acc64 = nullptr;
  int2* d_sort_rp = nullptr;
  float* d_sort_v = nullptr;
  int64_t *d_sort_hist = nullptr, *d_sort_flag = nullptr;
  int64_t sort_cap = 0, sort_cap2 = 0, sort_hist_cap = 0, sort_flag_cap = 0;
  float* d_cand_P = nullptr;
  double* d_T64 = nullptr;
  unsigned long long* d_cand_key = nullptr;
  float4* d_part = nullptr;
  float2* d_acc = nullptr;  // interleaved (model, weight) accumulators
  double *d_lse = nullptr, *d_plogp = nullptr;
  float* d_Tpart = nullptr;
  CUtensorMap tmKh, tmKt, tmBhi, tmBlo, tmPhi, tmPlo;
  CUtensorMap tmKh64, tmBhi64, tmBlo64, tmKt128;  // boxes of the two-SM contractions
  TcStatus* d_status = nullptr;
  // profiling: events at stage boundaries, kernel launch count
  // learned proposal: rotation cells and the candidate-iteration buffers
  int32_t n_cells = 0, cand_m = 0;
  // responsibilities of the last maximize: 1 dense, 2 proposed, 3 dense over
  // rotation chunks (kept as candidates)
  int resp_source = 0;
  float* d_cmass = nullptr;
  cudaEvent_t ev_sel = nullptr;  // the proposed iteration's selection has reached the host
  int32_t* d_best = nullptr;  // orientation diagnostics: most probable rotation per pattern
  float* d_bestp = nullptr;
  int64_t max_members = 0;
  std::vector<int64_t> h_mbeg;
  std::vector<int32_t> h_mcnt;
  int32_t* d_cell = nullptr;
  int64_t* d_mbeg = nullptr;
  int32_t* d_mcnt = nullptr;
  int32_t *d_cand = nullptr, *d_gpair = nullptr, *d_gcnt = nullptr;
  int64_t *d_ppos = nullptr, *d_gbeg = nullptr, *d_goff = nullptr;
  float *d_mass = nullptr, *d_Yc = nullptr, *d_Pt = nullptr;
  int4 *d_mtiles = nullptr, *d_ctiles = nullptr;
  TileDesc *d_gmt = nullptr, *d_gct = nullptr;   // tcgen05 grouped tile lists
  __half *d_Kg = nullptr, *d_Ahi = nullptr, *d_Alo = nullptr;
  // capacities (elements) of the per-iteration proposal buffers
  int64_t mtiles_cap = 0, ctiles_cap = 0, gmt_cap = 0, gct_cap = 0, pairs_cap = 0, slots_cap = 0,
          yc_cap = 0, pt_cap = 0, kg_cap = 0, a_ld = 0;
  double *d_lse_c = nullptr, *d_plogp_c = nullptr;
  float* d_lcmass = nullptr;  // [N][m] log responsibility mass of each candidate cell
  // responsibility lists of the mixed compress: per rotation the patterns with
  // a non-zero compress operand entry (offsets d_lrowoff [R+1]) and the entry
  unsigned long long* d_lcount = nullptr;  // entries compacted by the row-sum sweep
  int2* d_lcomp_rp = nullptr;              // their (rotation, pattern)
  float* d_lcomp_P = nullptr;              // and P
  int64_t lcomp_cap = 0, lcomp_cap2 = 0;
  int64_t *d_lrowtot = nullptr, *d_lrowoff = nullptr, *d_lcursor = nullptr;
  int32_t* d_lpat = nullptr;
  float* d_lx = nullptr;
  int64_t lcap = 0, lcap_x = 0, list_nnz = 0;
  bool list_mode = false;  // this iteration's compress reads the lists
  GroupArgs last_group{};     // arguments of the last grouped iteration (responsibility export)
  // dense audit of sampled patterns in a proposed iteration
  int64_t* d_aud_pat = nullptr;
  int32_t* d_aud_slot = nullptr;
  float *d_aud_scal = nullptr, *d_aud_cap = nullptr, *d_aud_K32 = nullptr, *d_aud_Y = nullptr;
  double *d_aud_patsq = nullptr, *d_aud_LL = nullptr;
  __half* d_aud_K16 = nullptr;
  float4* d_aud_part = nullptr;
  CUtensorMap tm_aud;
  int64_t audit_round = 0;
  cudaEvent_t ev_audit = nullptr;
  // Two event sets alternate between iterations, so the times of iteration
  // i-1 can be read while iteration i is still queued.
  // raster bands of the maximize / compress tile orders and the SM-pair forms
  // (defaults from measurements at 64^3 and 128^3, set per shape in
  // alloc_work; emc_autotune re-measures)
  emc_tuning tune{1, 6, 0, 0, 0, 0};
  // photon-list forms (FP32): the counts' non-zero entries by pattern (csr,
  // for the log-likelihood, with log W pixel-major in d_ST) and by active pixel
  // (csc, for the slice sums, with its entries divided by the scaling in aux
  // and the responsibilities pattern-major in d_PT); rebuilt after an upload
  SparseRows csr, csc;
  float* d_ST = nullptr;
  float* d_PT = nullptr;
  bool prof = false;
  cudaEvent_t ev[2][6] = {{nullptr}};
  int cur = 0;
  int64_t prof_iters = 0;
  int64_t launches = 0;
  void mark(int i) {
    if (!prof) return;
    if (i == 0) {
      cur ^= 1;
      ++prof_iters;
    }
    cudaEventRecord(ev[cur][i], st);
  }

  // pinned host staging of the proposed iteration, reused between calls
  void* hpin[8] = {nullptr};
  size_t hcap[8] = {0};
  template <class T>
  T* pinned(int slot, size_t n) {
    const size_t bytes = n * sizeof(T) + 16;
    if (bytes > hcap[slot]) {
      if (hpin[slot]) cudaFreeHost(hpin[slot]);
      hpin[slot] = nullptr;
      hcap[slot] = 0;
      const size_t b = bytes + bytes / 4 + 4096;
      if (cudaMallocHost(&hpin[slot], b) != cudaSuccess) return nullptr;
      hcap[slot] = b;
    }
    return static_cast<T*>(hpin[slot]);
  }

  emc_status fail(emc_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    err = buf;
    return s;
  }
  emc_status cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return EMC_OK;
    return fail(e == cudaErrorMemoryAllocation ? EMC_ERR_OOM : EMC_ERR_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
  }
  template <class T>
  emc_status alloc(T** p, size_t count, bool zero = false) {
    void* q = nullptr;
    const size_t bytes = count * sizeof(T) ? count * sizeof(T) : 16;
    if (mem_limit && mem_used + bytes > mem_limit)
      return fail(EMC_ERR_OOM, "device memory limit of %zu bytes reached (%zu held, %zu requested)",
                  mem_limit, mem_used, bytes);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return cuda(e, "cudaMalloc");
    allocs.push_back(q);
    alloc_bytes.push_back(bytes);
    mem_used += bytes;
    if (zero) {
      e = cudaMemsetAsync(q, 0, bytes, st);
      if (e != cudaSuccess) return cuda(e, "cudaMemset");
    }
    *p = static_cast<T*>(q);
    return EMC_OK;
  }
  void release(void* p) {
    for (size_t k = 0; k < allocs.size(); ++k)
      if (allocs[k] == p) {
        cudaFree(allocs[k]);
        allocs[k] = nullptr;
        mem_used -= alloc_bytes[k];
        alloc_bytes[k] = 0;
      }
  }
};

#define TRY(x)                              \
  do {                                      \
    emc_status _s = (x);                    \
    if (_s != EMC_OK) return _s;            \
  } while (0)
#define CK(ctx, x) TRY((ctx)->cuda((x), #x))

static thread_local std::string g_create_err;

// Number of entries of a host array that are NaN or infinite (or negative,
// when nonneg is set).
static int64_t count_bad(const float* x, int64_t n, bool nonneg) {
  int64_t bad = 0;
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(x[i]) || (nonneg && x[i] < 0.0f)) ++bad;
  return bad;
}


extern "C" {

static size_t avail_bytes(emc_context* c, size_t held);
static int64_t fit_rows(const emc_context* c, size_t bytes);
static emc_status set_y_rows(emc_context* c, int64_t rows);

const char* emc_status_string(emc_status s) {
  switch (s) {
    case EMC_OK: return "ok";
    case EMC_ERR_ARG: return "invalid argument";
    case EMC_ERR_CUDA: return "CUDA error";
    case EMC_ERR_OOM: return "out of device memory";
    case EMC_ERR_TIMEOUT: return "device wait timed out";
    case EMC_ERR_STATE: return "call out of order";
    case EMC_ERR_RANGE: return "data outside the exact range of the selected precision";
    case EMC_ERR_UNSUPPORTED: return "unsupported";
  }
  return "unknown status";
}

const char* emc_last_error(const emc_context* ctx) {
  return ctx ? ctx->err.c_str() : g_create_err.c_str();
}

emc_status emc_create(const emc_config* cfg, emc_context** out) {
  if (!cfg || !out) return EMC_ERR_ARG;
  *out = nullptr;
  if (cfg->side < 2 || cfg->side > 1024 || cfg->n_patterns < 1 || cfg->n_rotations < 1 ||
      (cfg->likelihood != EMC_LL_GAUSS && cfg->likelihood != EMC_LL_POISSON) ||
      (cfg->interp != EMC_INTERP_NEAREST && cfg->interp != EMC_INTERP_TRILINEAR) ||
      (cfg->precision != EMC_PREC_FP32 && cfg->precision != EMC_PREC_MIXED) ||
      (cfg->likelihood == EMC_LL_GAUSS && !(cfg->sigma > 0)) ||
      (cfg->likelihood == EMC_LL_POISSON && !(cfg->poisson_floor > 0))) {
    g_create_err = "emc_create: invalid configuration";
    return EMC_ERR_ARG;
  }
  emc_context* c = new emc_context();
  c->cfg = *cfg;
  c->N = cfg->n_patterns;
  c->R = cfg->n_rotations;
  c->npix = (int64_t)cfg->side * cfg->side;
  c->M = c->npix * cfg->side;
  c->mixed = cfg->precision == EMC_PREC_MIXED;
  c->gauss = cfg->likelihood == EMC_LL_GAUSS;
  auto bail = [&](emc_status s) {
    g_create_err = c->err;
    emc_destroy(c);
    return s;
  };
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) return bail(c->cuda(e, "cudaSetDevice"));
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, cfg->device);
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, cfg->device);
  if (c->mixed && major != 10) {
    c->fail(EMC_ERR_UNSUPPORTED, "mixed precision needs an sm_100 device (found sm_%d)", major * 10);
    return bail(EMC_ERR_UNSUPPORTED);
  }
  e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(c->cuda(e, "cudaStreamCreate"));
  emc_status s;
  // model and weight are adjacent: on the FP32 path they are the insertion
  // accumulators, reduced across ranks as one buffer of 2*M floats
  if ((s = c->alloc(&c->d_model, 2 * c->M, true)) ||
      (s = c->alloc(&c->d_scaling, c->N)) || (s = c->alloc(&c->d_scaling_prev, c->N)) ||
      (s = c->alloc(&c->d_quat, 4 * c->R)) || (s = c->alloc(&c->d_rotw, c->R)) ||
      (s = c->alloc(&c->d_T, c->R, true)) || (s = c->alloc(&c->d_Tskip, c->R, true)) ||
      (s = c->alloc(&c->d_rowstat, c->R, true)) ||
      (s = c->alloc(&c->d_scratch, 4096)) || (s = c->alloc(&c->d_stats, 16, true)) ||
      (s = c->alloc(&c->d_patsq, c->N, true)) || (s = c->alloc(&c->d_patsum, c->N, true)) ||
      (s = c->alloc(&c->d_status, 1, true)))
    return bail(s);
  c->d_weight = c->d_model + c->M;
  if ((s = c->cuda(launch_fill(c->d_scaling, c->N, 1.0f, c->st), "fill")) != EMC_OK) return bail(s);
  *out = c;
  return EMC_OK;
}

emc_status emc_destroy(emc_context* ctx) {
  if (!ctx) return EMC_OK;
  if (ctx->st) cudaStreamSynchronize(ctx->st);
  for (void* p : ctx->allocs)
    if (p) cudaFree(p);
  for (auto& set : ctx->ev)
    for (auto& e : set)
      if (e) cudaEventDestroy(e);
  for (void* h : ctx->hpin)
    if (h) cudaFreeHost(h);
  if (ctx->ev_sel) cudaEventDestroy(ctx->ev_sel);
  if (ctx->ev_audit) cudaEventDestroy(ctx->ev_audit);
  if (ctx->st) cudaStreamDestroy(ctx->st);
  delete ctx;
  return EMC_OK;
}

void* emc_stream(emc_context* ctx) { return ctx ? (void*)ctx->st : nullptr; }
int64_t emc_launch_count(const emc_context* ctx) { return ctx ? ctx->launches : 0; }

emc_status emc_set_memory_limit(emc_context* c, size_t bytes) {
  if (!c) return EMC_ERR_ARG;
  if (bytes && bytes < c->mem_used)
    return c->fail(EMC_ERR_ARG, "limit %zu is below the %zu bytes already held", bytes,
                   c->mem_used);
  c->mem_limit = bytes;
  return EMC_OK;
}

size_t emc_memory_used(const emc_context* c) { return c ? c->mem_used : 0; }

emc_status emc_set_rotation_chunk(emc_context* c, int64_t rows, int64_t capacity) {
  if (!c || rows < -1 || capacity < 0) return EMC_ERR_ARG;
  if (!c->mixed) return c->fail(EMC_ERR_UNSUPPORTED, "rotation chunks are a form of the mixed path");
  if (!c->have_geom) return c->fail(EMC_ERR_STATE, "set the geometry first");
  if (c->stage != 0 || c->batched)
    return c->fail(EMC_ERR_STATE, "rotation chunks change between iterations, outside a batch");
  const int64_t R = c->R;
  if (rows == -1) {
    // what Y and P' hold now is given back first
    size_t held = sizeof(float) * (size_t)(c->y_rows * c->Npad);
    if (c->d_Phi) held += 4 * (size_t)(c->Rpad * c->Npad);
    rows = fit_rows(c, avail_bytes(c, held) / 2);
  } else if (rows == 0) {
    rows = R;
  } else if (rows < R && rows % 256) {
    return c->fail(EMC_ERR_ARG, "a rotation chunk is a multiple of 256 rotations");
  }
  if (rows < R && c->npa > kListMaxPixels)
    return c->fail(EMC_ERR_UNSUPPORTED,
                   "rotation chunks need the responsibility lists (at most %d active pixels)",
                   kListMaxPixels);
  c->cand_cap_min = capacity;
  TRY(set_y_rows(c, rows));
  if (rows < R) c->tune.compress_sparse = 1;
  return EMC_OK;
}

int64_t emc_rotation_chunk(const emc_context* c) { return c ? c->y_rows : 0; }

emc_status emc_set_deterministic(emc_context* c, int on) {
  if (!c || (on != 0 && on != 1)) return EMC_ERR_ARG;
  if (c->stage != 0 || c->batched)
    return c->fail(EMC_ERR_STATE, "the insertion mode changes between iterations, outside a batch");
  if (on && !c->d_acc64) TRY(c->alloc(&c->d_acc64, 8 * c->M));
  c->det = on != 0;
  return EMC_OK;
}

emc_status emc_set_profiling(emc_context* c, int on) {
  if (!c) return EMC_ERR_ARG;
  if (on && !c->ev[0][0])
    for (auto& set : c->ev)
      for (auto& e : set) CK(c, cudaEventCreate(&e));
  c->prof = on != 0;
  c->prof_iters = 0;
  return EMC_OK;
}

emc_status emc_stage_times(emc_context* c, float* ms) {
  // times of the previous profiled iteration when there is one (the newest
  // may still be running), else of the newest
  if (!c || !ms) return EMC_ERR_ARG;
  if (!c->ev[0][0] || c->prof_iters == 0) return c->fail(EMC_ERR_STATE, "nothing profiled");
  const int set = c->prof_iters >= 2 ? (c->cur ^ 1) : c->cur;
  CK(c, cudaEventSynchronize(c->ev[set][5]));
  for (int i = 0; i < 5; ++i)
    CK(c, cudaEventElapsedTime(&ms[i], c->ev[set][i], c->ev[set][i + 1]));
  return EMC_OK;
}
int64_t emc_active_pixels(const emc_context* ctx) { return ctx ? ctx->npa : 0; }

// Device bytes this context may still allocate, after `held` bytes it holds
// are given back, less a reserve for the pattern staging, the photon and
// responsibility lists and scratch.
static size_t avail_bytes(emc_context* c, size_t held) {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 0;
  size_t a = fr + held;
  if (c->mem_limit) {
    const size_t used = c->mem_used - held;
    a = std::min(a, c->mem_limit > used ? c->mem_limit - used : 0);
  }
  const size_t reserve =
      sizeof(float) * (size_t)c->N * (size_t)(c->npix + c->npa) + ((size_t)1 << 30);
  return a > reserve ? a - reserve : 0;
}

// The most rotations (a multiple of 256, at least 256) whose Y fits in `bytes`.
static int64_t fit_rows(const emc_context* c, size_t bytes) {
  const int64_t rows = (int64_t)(bytes / (sizeof(float) * (size_t)c->Npad)) / 256 * 256;
  return rows < 256 ? 256 : rows;
}

// Y for `rows` rotations (a multiple of 256, or R and more: every rotation).
// Chunks drop the dense compress operand P', which only the unchunked
// maximize writes; one chunk of every rotation allocates it again.
static emc_status set_y_rows(emc_context* c, int64_t rows) {
  if (rows >= c->R) rows = c->R;
  if (c->d_Y && rows == c->y_rows) return EMC_OK;
  if (c->d_Y) c->release(c->d_Y);
  c->d_Y = nullptr;
  c->y_rows = 0;
  c->resp_source = 0;  // the last iteration's responsibilities are gone with Y
  if (rows < c->R)
    for (__half** q : {&c->d_Phi, &c->d_Plo})
      if (*q) {
        c->release(*q);
        *q = nullptr;
      }
  TRY(c->alloc(&c->d_Y, rows * c->Npad));
  if (rows == c->R && !c->d_Phi) {
    TRY(c->alloc(&c->d_Phi, c->Rpad * c->Npad, true));
    TRY(c->alloc(&c->d_Plo, c->Rpad * c->Npad, true));
    if (!tc_encode_2d(&c->tmPhi, c->d_Phi, c->Npad, c->Rpad, 128, kCompressBK) ||
        !tc_encode_2d(&c->tmPlo, c->d_Plo, c->Npad, c->Rpad, 128, kCompressBK))
      return c->fail(EMC_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  }
  c->y_rows = rows;
  return EMC_OK;
}

static emc_status alloc_work(emc_context* c) {
  // called once geometry is known (npa fixes every pixel dimension)
  const int64_t R = c->R, N = c->N, npa = c->npa;
  if (c->cfg.interp == EMC_INTERP_TRILINEAR)
    TRY(c->alloc(&c->d_tri, tri_table_entries(c->cfg.side)));
  if (!c->mixed) {
    TRY(c->alloc(&c->d_S, R * npa));
    TRY(c->alloc(&c->d_LL, R * N));
    // the log-likelihood is kept in FP64: its values reach 10^3 - 10^4 (poisson),
    // where an FP32 ulp (1e-4 - 1e-3) would move the responsibilities by more
    // than the contraction's own error
    TRY(c->alloc(&c->d_LL64, R * N));
    TRY(c->alloc(&c->d_K, N * npa));
    TRY(c->alloc(&c->d_den, ((R + 127) / 128) * N));
    TRY(c->alloc(&c->d_plogp_part, (N + 31) / 32 + 1));
    TRY(c->alloc(&c->d_lse32, N));
    return EMC_OK;
  }
  c->Npad = round_up(N, 128);
  c->Ppad = round_up(npa, 256);
  // the two-SM maximize pays where the pixel extent is long (measured: 18%
  // faster at 16,384 padded pixels, 8% slower at 4,096); emc_autotune decides
  c->tune.maximize_pair = c->Ppad >= 8192 ? 1 : 0;
  // the compress on pairs: 5% faster at 128^3 / 50k patterns (raster 2)
  c->tune.compress_pair = (c->Ppad >= 8192 && c->Npad >= 8192) ? 1 : 0;
  // the compress from responsibility lists (a handful of non-zero entries
  // per pattern once the posteriors are sharp) where its shared-memory slice fits
  c->tune.compress_sparse = npa <= kListMaxPixels ? 1 : 0;
  if (c->tune.compress_pair) c->tune.compress_raster = 2;
  c->Rpad = round_up(R, 256);
  c->nrt = c->Rpad / 256;
  TRY(c->alloc(&c->d_acc, c->M, true));
  // the nearest expansion's voxel table (here rather than at the first
  // expansion, so an iteration can be captured into a graph before any ran)
  if (c->cfg.interp == EMC_INTERP_NEAREST) TRY(c->alloc(&c->d_vtab, c->M + 1));
  TRY(c->alloc(&c->d_Kh, c->Npad * c->Ppad, true));
  TRY(c->alloc(&c->d_Kt, c->Ppad * c->Npad, true));
  TRY(c->alloc(&c->d_Bhi, c->Rpad * c->Ppad, true));
  TRY(c->alloc(&c->d_Blo, c->Rpad * c->Ppad, true));
  TRY(c->alloc(&c->d_part, c->nrt * N));
  TRY(c->alloc(&c->d_lse, N));
  TRY(c->alloc(&c->d_plogp, N));
  TRY(c->alloc(&c->d_Tpart, ((N + 1023) / 1024) * R));
  // Y (R x Npad FP32) and the dense compress operand P' (2 x Rpad x Npad
  // FP16) are the large buffers.  Where they do not fit the memory limit or
  // the free device memory, Y holds rotation chunks (half of what is left)
  // and P' is not kept: the compress reads responsibility lists.
  const size_t full = sizeof(float) * (size_t)(R * c->Npad) + 4 * (size_t)(c->Rpad * c->Npad);
  const size_t avail = avail_bytes(c, 0);
  int64_t rows = R;
  if (full > avail && c->tune.compress_sparse) rows = fit_rows(c, avail / 2);
  TRY(set_y_rows(c, rows));
  bool ok = tc_encode_2d(&c->tmKh, c->d_Kh, c->Ppad, c->Npad, 128, kMaximizeBK) &&
            tc_encode_2d(&c->tmBhi, c->d_Bhi, c->Ppad, c->Rpad, 256, kMaximizeBK) &&
            tc_encode_2d(&c->tmBlo, c->d_Blo, c->Ppad, c->Rpad, 256, kMaximizeBK) &&
            tc_encode_2d(&c->tmKt, c->d_Kt, c->Npad, c->Ppad, 256, kCompressBK) &&
            tc_encode_2d(&c->tmKh64, c->d_Kh, c->Ppad, c->Npad, 128, kPairBoxK) &&
            tc_encode_2d(&c->tmBhi64, c->d_Bhi, c->Ppad, c->Rpad, 128, kPairBoxK) &&
            tc_encode_2d(&c->tmBlo64, c->d_Blo, c->Ppad, c->Rpad, 128, kPairBoxK) &&
            tc_encode_2d(&c->tmKt128, c->d_Kt, c->Npad, c->Ppad, 128, kPairBoxK);
  if (!ok) return c->fail(EMC_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return EMC_OK;
}

emc_status emc_set_geometry(emc_context* c, const float* x, const float* y, const float* z,
                            const int32_t* mask) {
  if (!c || !x || !y || !z || !mask) return EMC_ERR_ARG;
  if (c->have_geom) return c->fail(EMC_ERR_STATE, "geometry is already set");
  if (count_bad(x, c->npix, false) || count_bad(y, c->npix, false) || count_bad(z, c->npix, false))
    return c->fail(EMC_ERR_RANGE, "pixel coordinates must be finite");
  std::vector<int32_t> pix, ins;
  std::vector<float> cx, cy, cz;
  for (int64_t i = 0; i < c->npix; ++i)
    if (mask[i] != 0) {  // emc_cuda.cu:120: pixels with mask != 0 enter the likelihood
      pix.push_back((int32_t)i);
      ins.push_back(mask[i] == 1 ? 1 : 0);  // emc_atomic.cu:30: only mask == 1 is inserted
      cx.push_back(x[i]);
      cy.push_back(y[i]);
      cz.push_back(z[i]);
    }
  if (pix.empty()) return c->fail(EMC_ERR_ARG, "mask has no active pixel");
  c->npa = (int64_t)pix.size();
  std::vector<int32_t> rank;
  if (c->mixed) {
    // The mixed path's operands list the active pixels along a Morton
    // (Z-order) curve of the detector: consecutive pixels then form compact
    // patches, whose voxels under any rotation lie close together, so the
    // expansion's gathers and the insertion's atomics of a warp touch fewer
    // cache sectors.  The pixel order of a contraction is free; rank[j] is
    // pixel j's position in the ascending order, which the slice export uses.
    auto morton = [](uint32_t x, uint32_t y) {
      uint64_t k = 0;
      for (int b = 0; b < 16; ++b)
        k |= ((uint64_t)((x >> b) & 1u) << (2 * b)) | ((uint64_t)((y >> b) & 1u) << (2 * b + 1));
      return k;
    };
    std::vector<int32_t> ord(pix.size());
    for (size_t j = 0; j < ord.size(); ++j) ord[j] = (int32_t)j;
    const int side = c->cfg.side;
    std::stable_sort(ord.begin(), ord.end(), [&](int32_t a, int32_t b) {
      return morton(pix[a] % side, pix[a] / side) < morton(pix[b] % side, pix[b] / side);
    });
    auto permute = [&](auto& v) {
      auto w = v;
      for (size_t j = 0; j < ord.size(); ++j) w[j] = v[ord[j]];
      v.swap(w);
    };
    permute(pix);
    permute(ins);
    permute(cx);
    permute(cy);
    permute(cz);
    rank = ord;
  }
  TRY(c->alloc(&c->d_pix, c->npa));
  TRY(c->alloc(&c->d_ins, c->npa));
  TRY(c->alloc(&c->d_cx, c->npa));
  TRY(c->alloc(&c->d_cy, c->npa));
  TRY(c->alloc(&c->d_cz, c->npa));
  CK(c, cudaMemcpyAsync(c->d_pix, pix.data(), 4 * c->npa, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_ins, ins.data(), 4 * c->npa, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_cx, cx.data(), 4 * c->npa, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_cy, cy.data(), 4 * c->npa, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_cz, cz.data(), 4 * c->npa, cudaMemcpyHostToDevice, c->st));
  if (!rank.empty()) {
    TRY(c->alloc(&c->d_rank, c->npa));
    CK(c, cudaMemcpyAsync(c->d_rank, rank.data(), 4 * c->npa, cudaMemcpyHostToDevice, c->st));
  }
  TRY(alloc_work(c));
  CK(c, cudaStreamSynchronize(c->st));
  c->have_geom = true;
  return EMC_OK;
}

emc_status emc_set_rotations(emc_context* c, const float* q, const float* w) {
  if (!c || !q || !w) return EMC_ERR_ARG;
  if (count_bad(q, 4 * c->R, false) || count_bad(w, c->R, true))
    return c->fail(EMC_ERR_RANGE, "rotations must be finite and their weights non-negative");
  CK(c, cudaMemcpyAsync(c->d_quat, q, sizeof(float) * 4 * c->R, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_rotw, w, sizeof(float) * c->R, cudaMemcpyHostToDevice, c->st));
  c->have_rot = true;
  return EMC_OK;
}

static emc_status finish_patterns(emc_context* c);

emc_status emc_set_patterns(emc_context* c, const float* counts) {
  if (!c || !counts) return EMC_ERR_ARG;
  if (!c->have_geom) return c->fail(EMC_ERR_STATE, "set the geometry before the patterns");
  const int64_t N = c->N, npa = c->npa;
  // full images to the device, then gathered to the active pixels there;
  // the staging buffers are allocated on the first call and kept
  if (!c->d_stage) TRY(c->alloc(&c->d_stage, N * c->npix));
  if (c->mixed && !c->d_K) TRY(c->alloc(&c->d_K, N * npa));
  float* full = c->d_stage;
  float* compact = c->d_K;
  cudaError_t e = cudaMemcpyAsync(full, counts, sizeof(float) * N * c->npix,
                                  cudaMemcpyHostToDevice, c->st);
  if (e == cudaSuccess) {
    for (int64_t r0 = 0; r0 < N && e == cudaSuccess; r0 += 65535) {
      const int64_t rows = N - r0 < 65535 ? N - r0 : 65535;
      gather_cols_kernel<<<dim3(8, (unsigned)rows), 256, 0, c->st>>>(full + r0 * c->npix, rows,
                                                                      c->npix, c->d_pix, npa,
                                                                      compact + r0 * npa);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) return c->cuda(e, "emc_set_patterns");
  return finish_patterns(c);
}

// Pattern statistics and the FP16 operands of the compact counts d_K.
static emc_status finish_patterns(emc_context* c) {
  const int64_t N = c->N, npa = c->npa;
  float* compact = c->d_K;
  cudaError_t e = launch_pattern_stats(compact, nullptr, N, npa, npa, 1, c->d_patsq, c->st);
  if (e == cudaSuccess) e = launch_pattern_stats(compact, nullptr, N, npa, npa, 0, c->d_patsum, c->st);
  int bad = 0;
  int* d_bad = reinterpret_cast<int*>(c->d_scratch);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, sizeof(int), c->st);
  if (e == cudaSuccess && c->mixed)
    e = launch_pack_patterns(compact, N, npa, c->Npad, c->Ppad, c->d_Kh, c->d_Kt, d_bad, c->st);
  else if (e == cudaSuccess)
    e = launch_count_invalid(compact, N * npa, d_bad, c->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  if (e != cudaSuccess) return c->cuda(e, "emc_set_patterns");
  c->have_pat = false;
  if (bad && c->mixed)
    return c->fail(EMC_ERR_RANGE,
                   "%d counts are not integers in [0, 2048]; the mixed path needs them exact in FP16",
                   bad);
  if (bad)
    return c->fail(EMC_ERR_RANGE, "%d counts are negative, NaN or infinite", bad);
  c->have_pat = true;
  c->csr.valid = false;
  c->csc.valid = false;
  return EMC_OK;
}

emc_status emc_set_patterns_sparse(emc_context* c, const int64_t* row_ptr, const int32_t* pixels,
                                   const float* counts) {
  if (!c || !row_ptr) return EMC_ERR_ARG;
  if (!c->have_geom) return c->fail(EMC_ERR_STATE, "set the geometry before the patterns");
  const int64_t N = c->N, npa = c->npa;
  const int64_t nnz = row_ptr[N];
  if (row_ptr[0] != 0 || nnz < 0 || (nnz > 0 && !pixels))
    return c->fail(EMC_ERR_ARG, "row_ptr must start at 0 and end at the entry count");
  for (int64_t p = 0; p < N; ++p)
    if (row_ptr[p + 1] < row_ptr[p]) return c->fail(EMC_ERR_ARG, "row_ptr must not decrease");
  if (!c->d_compact_of) {
    std::vector<int32_t> inv(c->npix, -1);
    std::vector<int32_t> pix(npa);
    CK(c, cudaMemcpyAsync(pix.data(), c->d_pix, sizeof(int32_t) * npa, cudaMemcpyDeviceToHost, c->st));
    CK(c, cudaStreamSynchronize(c->st));
    for (int64_t j = 0; j < npa; ++j) inv[pix[j]] = (int32_t)j;
    TRY(c->alloc(&c->d_compact_of, c->npix));
    CK(c, cudaMemcpyAsync(c->d_compact_of, inv.data(), sizeof(int32_t) * c->npix,
                          cudaMemcpyHostToDevice, c->st));
  }
  if (!c->d_K) TRY(c->alloc(&c->d_K, N * npa));
  if (!c->d_sp_row) TRY(c->alloc(&c->d_sp_row, N + 1));
  if (nnz > c->sp_cap) {
    for (void* q : {(void*)c->d_sp_pix, (void*)c->d_sp_val})
      if (q) c->release(q);
    c->d_sp_pix = nullptr;
    c->d_sp_val = nullptr;
    c->sp_cap = 0;
    const int64_t cap = nnz + nnz / 4 + 1024;
    TRY(c->alloc(&c->d_sp_pix, cap));
    TRY(c->alloc(&c->d_sp_val, cap));
    c->sp_cap = cap;
  }
  CK(c, cudaMemcpyAsync(c->d_sp_row, row_ptr, sizeof(int64_t) * (N + 1), cudaMemcpyHostToDevice, c->st));
  if (nnz > 0) {
    CK(c, cudaMemcpyAsync(c->d_sp_pix, pixels, sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, c->st));
    if (counts)
      CK(c, cudaMemcpyAsync(c->d_sp_val, counts, sizeof(float) * nnz, cudaMemcpyHostToDevice, c->st));
  }
  int* d_bad = reinterpret_cast<int*>(c->d_scratch) + 1;
  int bad = 0;
  CK(c, cudaMemsetAsync(d_bad, 0, sizeof(int), c->st));
  CK(c, cudaMemsetAsync(c->d_K, 0, sizeof(float) * N * npa, c->st));
  scatter_photons_kernel<<<(unsigned)((N + 7) / 8), 256, 0, c->st>>>(
      c->d_sp_row, c->d_sp_pix, counts ? c->d_sp_val : nullptr, N, c->npix, c->d_compact_of, npa,
      c->d_K, d_bad);
  CK(c, cudaGetLastError());
  CK(c, cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  if (bad) return c->fail(EMC_ERR_ARG, "%d photon entries lie outside the detector", bad);
  return finish_patterns(c);
}

emc_status emc_set_model(emc_context* c, const float* model) {
  if (!c || !model) return EMC_ERR_ARG;
  if (const int64_t b = count_bad(model, c->M, false))
    return c->fail(EMC_ERR_RANGE, "%lld model values are NaN or infinite", (long long)b);
  CK(c, cudaMemcpyAsync(c->d_model, model, sizeof(float) * c->M, cudaMemcpyHostToDevice, c->st));
  c->have_model = true;
  c->stage = 0;
  return EMC_OK;
}

emc_status emc_set_scaling(emc_context* c, const float* scaling) {
  if (!c || !scaling) return EMC_ERR_ARG;
  for (int64_t p = 0; p < c->N; ++p)
    if (!(scaling[p] > 0.0f) || !std::isfinite(scaling[p]))
      return c->fail(EMC_ERR_RANGE, "scaling of pattern %lld is not a finite positive number",
                     (long long)p);
  CK(c, cudaMemcpyAsync(c->d_scaling, scaling, sizeof(float) * c->N, cudaMemcpyHostToDevice, c->st));
  return EMC_OK;
}

static double gauss_inv(const emc_context* c) {
  return 1.0 / (2.0 * (double)c->npa * (double)c->cfg.sigma * (double)c->cfg.sigma);
}

emc_status emc_expand(emc_context* c) {
  StageRange range("emc expand");
  if (!c) return EMC_ERR_ARG;
  if (!c->have_geom || !c->have_rot || !c->have_pat || !c->have_model)
    return c->fail(EMC_ERR_STATE, "geometry, rotations, patterns and model must be set first");
  if (c->stage != 0) return c->fail(EMC_ERR_STATE, "expand called out of order");
  ExpandArgs a{};
  a.model = c->d_model;
  a.quat = c->d_quat;
  a.cx = c->d_cx;
  a.cy = c->d_cy;
  a.cz = c->d_cz;
  a.R = c->R;
  a.npix = c->npa;
  a.side = c->cfg.side;
  a.interp = c->cfg.interp;
  a.floor_ = c->cfg.poisson_floor;
  a.rowstat = c->d_rowstat;
  if (!c->mixed) {
    a.ld = c->npa;
    a.out = c->gauss ? EXP_F32 : EXP_LOG_F32;
    a.stat = c->gauss ? STAT_NONE : STAT_SUM;
    a.out_f32 = c->d_S;
  } else {
    a.ld = c->Ppad;
    a.out = EXP_F16_SPLIT;
    a.log_split = c->gauss ? 0 : 1;
    a.stat = c->gauss ? STAT_SUMSQ : STAT_SUM;
    a.out_hi = c->d_Bhi;
    a.out_lo = c->d_Blo;
  }
  c->mark(0);
  if (c->mixed && c->cfg.interp == EMC_INTERP_NEAREST) {
    if (!c->d_vtab) TRY(c->alloc(&c->d_vtab, c->M + 1));
    CK(c, launch_expand_table(c->d_model, c->M, a.floor_, a.log_split, c->d_vtab, c->st));
    a.tab = c->d_vtab;
    c->launches += 1;
  }
  if (c->d_tri) {
    CK(c, launch_tri_table(c->d_model, c->cfg.side, c->d_tri, c->st));
    a.tri = c->d_tri;
    c->launches += 1;
  }
  CK(c, launch_expand(a, c->st));
  c->launches += 1;
  c->mark(1);
  c->stage = 1;
  return EMC_OK;
}

}  // extern "C"

// Epilogue arguments of the mixed maximize contraction.
static MaxEpiArgs max_args(emc_context* c) {
  MaxEpiArgs e{};
  e.N = c->N;
  e.R = c->R;
  e.ldY = c->Npad;
  e.poisson = c->gauss ? 0 : 1;
  e.scaling = c->d_scaling_prev;
  e.rowstat = c->d_rowstat;
  e.patstat = c->d_patsq;
  e.gauss_inv = gauss_inv(c);
  e.Y = c->d_Y;
  e.part = c->d_part;
  return e;
}

// Epilogue arguments of the mixed compress contraction (insertion).
static CmpEpiArgs cmp_args(emc_context* c) {
  CmpEpiArgs e{};
  e.R = c->R;
  e.npa = c->npa;
  e.side = c->cfg.side;
  e.interp = c->cfg.interp;
  e.inv_c0 = 1.0f;
  e.quat = c->d_quat;
  e.rotw = c->d_rotw;
  e.T = c->d_T;
  e.Tskip = c->d_Tskip;
  e.cx = c->d_cx;
  e.cy = c->d_cy;
  e.cz = c->d_cz;
  e.ins = c->d_ins;
  e.acc = c->d_acc;
  return e;
}

// After the maximize contraction: lse, new scaling and sum P log P per
// pattern, T_r, the compress operand P / (T_r phi), and the stats sums.
// Grows a work buffer to hold at least `need` elements (contents not kept).
template <class T>
static emc_status grow(emc_context* c, T** p, int64_t& cap, int64_t need) {
  if (need <= cap && *p) return EMC_OK;
  if (*p) c->release(*p);
  *p = nullptr;
  cap = 0;
  const int64_t n = need + need / 4 + 64;
  TRY(c->alloc(p, n));
  cap = n;
  return EMC_OK;
}


static emc_status build_rows(emc_context* c, const float* M, int64_t rows, int64_t cols,
                             SparseRows& s, bool with_aux);

// Arguments of the responsibility pass over every rotation.
static RespArgs resp_args(emc_context* c) {
  RespArgs a{};
  a.N = c->N;
  a.R = c->R;
  a.ldY = c->Npad;
  a.ldP = c->Npad;
  a.nparts = c->nrt;
  a.poisson = c->gauss ? 0 : 1;
  a.Y = c->d_Y;
  a.part = c->d_part;
  a.scaling = c->d_scaling_prev;
  a.rowstat = c->d_rowstat;
  a.patstat = c->d_patsq;
  a.patsum = c->d_patsum;
  a.gauss_inv = gauss_inv(c);
  a.lse = c->d_lse;
  a.plogp = c->d_plogp;
  a.new_scaling = c->d_scaling;
  a.c0 = 1.0f;
  a.Phi = c->d_Phi;
  a.Plo = c->d_Plo;
  a.Tpart = c->d_Tpart;
  a.T = c->d_T;
  a.P32 = nullptr;
  return a;
}

static emc_status list_buffers(emc_context* c) {
  if (!c->d_lcount) {
    const int64_t R = c->R;
    TRY(c->alloc(&c->d_lcount, 1));
    TRY(c->alloc(&c->d_lrowtot, R));
    TRY(c->alloc(&c->d_lrowoff, R + 1));
    TRY(c->alloc(&c->d_lcursor, R));
  }
  return EMC_OK;
}

// Room for `n` compacted (rotation, pattern, value) entries.
static emc_status compact_capacity(emc_context* c, int64_t n) {
  if (c->lcomp_cap >= n && c->d_lcomp_rp) return EMC_OK;
  int64_t cap = c->lcomp_cap;
  TRY(grow(c, &c->d_lcomp_rp, cap, n));
  int64_t cap2 = c->lcomp_cap2;
  TRY(grow(c, &c->d_lcomp_P, cap2, cap));
  c->lcomp_cap = cap;
  c->lcomp_cap2 = cap2;
  return EMC_OK;
}

// Scratch of the deterministic (rotation, pattern) sort of n entries.
static emc_status sort_scratch(emc_context* c, int64_t n) {
  TRY(grow(c, &c->d_sort_rp, c->sort_cap, n + 1));
  TRY(grow(c, &c->d_sort_v, c->sort_cap2, n + 1));
  TRY(grow(c, &c->d_sort_hist, c->sort_hist_cap, sort_hist_size(n)));
  TRY(grow(c, &c->d_sort_flag, c->sort_flag_cap, 2 * n + 2 + scan_scratch(n)));
  return EMC_OK;
}

static emc_status mixed_resp_pass(emc_context* c, bool allow_lists = true) {
  const int64_t N = c->N;
  RespArgs a = resp_args(c);
  c->list_mode = false;
  if (allow_lists && c->tune.compress_sparse && c->npa <= kListMaxPixels) {
    // the compress operand as per-rotation lists of its non-zero entries:
    // entries P >= kListMinP are compacted during the row-sum sweep, the host
    // reads their count (one wait), a counting sort orders them by rotation
    TRY(list_buffers(c));
    TRY(compact_capacity(c, std::max<int64_t>(64 * N, (int64_t)1 << 20)));
    CK(c, cudaMemsetAsync(c->d_lcount, 0, sizeof(unsigned long long), c->st));
    a.list_count = c->d_lcount;
    a.list_cap = c->lcomp_cap;
    a.list_rp = c->d_lcomp_rp;
    a.list_P = c->d_lcomp_P;
    a.list_min = kListMinP;
    CK(c, launch_resp_rowsums(a, c->st));
    unsigned long long* hn = c->pinned<unsigned long long>(7, 1);
    if (!hn) return c->fail(EMC_ERR_OOM, "pinned host staging");
    CK(c, cudaMemcpyAsync(hn, c->d_lcount, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          c->st));
    CK(c, cudaStreamSynchronize(c->st));
    c->list_nnz = (int64_t)*hn;
    if (c->list_nnz <= c->lcomp_cap) {
      TRY(grow(c, &c->d_lpat, c->lcap, c->list_nnz + 1));
      int64_t cap = c->lcap_x;
      TRY(grow(c, &c->d_lx, cap, c->list_nnz + 1));
      c->lcap_x = cap;
      if (c->det) {
        // the entries in (rotation, pattern) order, so the lists do not
        // depend on the order the sweep appended them
        TRY(sort_scratch(c, c->list_nnz));
        CK(c, launch_finish_T(c->d_Tpart, N, c->R, c->d_T, c->st));
        CK(c, launch_sort_entries(c->d_lcomp_rp, c->d_lcomp_P, c->list_nnz, N, c->R,
                                  c->d_sort_rp, c->d_sort_v, c->d_sort_hist, c->st));
        CK(c, launch_list_from_sorted(c->d_lcomp_rp, c->d_lcomp_P, c->list_nnz, c->R, c->d_T,
                                      c->d_scaling, kListRel, c->d_lrowtot, c->d_lrowoff,
                                      c->d_sort_flag, c->d_lpat, c->d_lx, c->st));
      } else {
        CK(c, launch_list_from_compact(a, c->list_nnz, kListRel, c->d_lrowtot, c->d_lcursor,
                                       c->d_lrowoff, c->d_lpat, c->d_lx, c->st));
      }
      c->list_mode = true;
      c->launches += 6;  // combine, row sums, T, count, scan, fill
    } else {
      // more entries than the compaction holds: the dense operand this time,
      // room for them next time
      CK(c, launch_resp_write(a, c->st));
      TRY(compact_capacity(c, c->list_nnz));
      c->launches += 3;
    }
  } else {
    CK(c, launch_resp_pass(a, c->st));
    c->launches += 3;  // combine, 2 sweeps
  }
  CK(c, launch_sum_f64(c->d_plogp, N, c->d_stats + 2, c->st));
  CK(c, launch_sum_f64(c->d_lse, N, c->d_stats + 3, c->st));
  c->launches += 2;
  return EMC_OK;
}

// The responsibility pass of a batched dataset with lists, in a form a CUDA
// graph can hold: the count of compacted entries stays on the device, the
// lists are built from it when it fits the compaction's capacity, and the
// dense compress operand is written only when it does not (write_kernel
// gated on the count), so the compress then runs from the lists or, gated
// the other way, as the dense contraction.  No host wait and no allocation:
// batch_lists_ready sized every buffer when the batch was made.
static emc_status gated_list_pass(emc_context* c) {
  RespArgs a = resp_args(c);
  c->list_mode = false;
  CK(c, cudaMemsetAsync(c->d_lcount, 0, sizeof(unsigned long long), c->st));
  a.list_count = c->d_lcount;
  a.list_cap = c->lcomp_cap;
  a.list_rp = c->d_lcomp_rp;
  a.list_P = c->d_lcomp_P;
  a.list_min = kListMinP;
  CK(c, launch_resp_rowsums(a, c->st));
  CK(c, launch_list_from_compact(a, c->lcomp_cap, kListRel, c->d_lrowtot, c->d_lcursor,
                                 c->d_lrowoff, c->d_lpat, c->d_lx, c->st, c->d_lcount));
  a.gate_count = c->d_lcount;
  a.gate_cap = c->lcomp_cap;
  CK(c, launch_resp_write(a, c->st));
  CK(c, launch_sum_f64(c->d_plogp, c->N, c->d_stats + 2, c->st));
  CK(c, launch_sum_f64(c->d_lse, c->N, c->d_stats + 3, c->st));
  c->launches += 9;  // combine, row sums, T, count, scan, fill, write, 2 sums
  return EMC_OK;
}

// The buffers of gated_list_pass and of the list compress: the compaction
// (room for at least `entries`), the lists at its capacity and the counts'
// photon lists.
static emc_status batch_lists_ready(emc_context* c, int64_t entries) {
  TRY(list_buffers(c));
  TRY(compact_capacity(c, entries));
  TRY(grow(c, &c->d_lpat, c->lcap, c->lcomp_cap + 1));
  int64_t cap = c->lcap_x;
  TRY(grow(c, &c->d_lx, cap, c->lcomp_cap + 1));
  c->lcap_x = cap;
  if (!c->csr.valid) TRY(build_rows(c, c->d_K, c->N, c->npa, c->csr, false));
  return EMC_OK;
}

// The maximize over rotation chunks of y_rows rotations, Y holding one chunk
// at a time.  Per chunk: the contraction into Y and the chunk's tile
// partials; the combine over the partials of the chunks so far (the running
// lse, a lower bound of the final one); the row-sum sweep keeping the
// candidates, the entries with P >= kListMinP under the running lse, which
// include every entry the unchunked pass compacts.  After the last chunk,
// whose combine covers every tile, lse, scaling and sum P log P are those of
// the unchunked pass; P of the candidates under it gives T_r and the
// responsibility lists.  More candidates than the arrays hold: they grow and
// the chunks run again (the contraction is deterministic).
static emc_status chunked_maximize(emc_context* c) {
  const int64_t R = c->R, N = c->N, rows = c->y_rows;
  if (!(c->tune.compress_sparse && c->npa <= kListMaxPixels))
    return c->fail(EMC_ERR_STATE, "rotation chunks need the compress from responsibility lists");
  TRY(list_buffers(c));
  if (!c->d_T64) TRY(c->alloc(&c->d_T64, R));
  TRY(compact_capacity(c, c->cand_cap_min > 0 ? c->cand_cap_min
                                              : std::max<int64_t>(64 * N, (int64_t)1 << 20)));
  unsigned long long* hn = c->pinned<unsigned long long>(7, 1);
  if (!hn) return c->fail(EMC_ERR_OOM, "pinned host staging");
  const bool pair = c->tune.maximize_pair != 0;
  RespArgs a = resp_args(c);
  a.Tpart = nullptr;
  a.list_count = c->d_lcount;
  a.list_min = kListMinP;
  a.list_store_y = 1;
  for (int attempt = 0;; ++attempt) {
    a.list_cap = c->lcomp_cap;
    a.list_rp = c->d_lcomp_rp;
    a.list_P = c->d_lcomp_P;
    CK(c, cudaMemsetAsync(c->d_lcount, 0, sizeof(unsigned long long), c->st));
    for (int64_t r0 = 0; r0 < R; r0 += rows) {
      const int64_t rc = std::min(rows, R - r0), rcp = round_up(rc, 256);
      // the chunk's rows of the slice operand (r0 is a multiple of 256)
      CUtensorMap th, tl;
      if (!tc_encode_2d(&th, c->d_Bhi + r0 * c->Ppad, c->Ppad, rcp, pair ? 128 : 256,
                        pair ? kPairBoxK : kMaximizeBK) ||
          !tc_encode_2d(&tl, c->d_Blo + r0 * c->Ppad, c->Ppad, rcp, pair ? 128 : 256,
                        pair ? kPairBoxK : kMaximizeBK))
        return c->fail(EMC_ERR_CUDA, "tensor map encoding failed");
      MaxEpiArgs e = max_args(c);
      e.R = rc;
      e.rowstat = c->d_rowstat + r0;
      e.part = c->d_part + (r0 / 256) * N;
      if (pair)
        CK(c, launch_maximize_pair_tc(c->tmKh64, th, tl, c->Npad, rcp, c->Ppad, e, c->d_status,
                                      c->num_sms, c->st, c->tune.maximize_raster));
      else
        CK(c, launch_maximize_tc(c->tmKh, th, tl, c->Npad, rcp, c->Ppad, e, c->d_status,
                                 c->num_sms, c->st, c->tune.maximize_raster));
      a.R = rc;
      a.rowstat = c->d_rowstat + r0;
      a.nparts = (r0 + rcp) / 256;
      a.list_r0 = r0;
      CK(c, launch_resp_rowsums(a, c->st));  // combine + candidate sweep
      c->launches += 3;
    }
    CK(c, cudaMemcpyAsync(hn, c->d_lcount, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          c->st));
    CK(c, cudaStreamSynchronize(c->st));
    c->cand_n = (int64_t)*hn;
    if (c->cand_n <= c->lcomp_cap) break;
    if (attempt) return c->fail(EMC_ERR_CUDA, "candidate count changed between identical passes");
    TRY(compact_capacity(c, c->cand_n));
  }
  c->mark(2);
  TRY(grow(c, &c->d_cand_P, c->cand_P_cap, c->cand_n + 1));
  TRY(grow(c, &c->d_lpat, c->lcap, c->cand_n + 1));
  int64_t cap = c->lcap_x;
  TRY(grow(c, &c->d_lx, cap, c->cand_n + 1));
  c->lcap_x = cap;
  a.R = R;
  a.rowstat = c->d_rowstat;
  a.list_r0 = 0;
  if (c->det) {
    // candidates in (rotation, pattern) order, then P, T_r summed in that
    // order and the lists in it
    TRY(sort_scratch(c, c->cand_n));
    CK(c, launch_sort_entries(c->d_lcomp_rp, c->d_lcomp_P, c->cand_n, N, R, c->d_sort_rp,
                              c->d_sort_v, c->d_sort_hist, c->st));
    CK(c, launch_cand_probs(a, c->cand_n, c->d_cand_P, c->d_T64, c->st));
    CK(c, launch_T_from_sorted(c->d_lcomp_rp, c->d_cand_P, c->cand_n, R, c->d_lrowtot,
                               c->d_lrowoff, c->d_T, c->st));
    CK(c, launch_list_from_sorted(c->d_lcomp_rp, c->d_cand_P, c->cand_n, R, c->d_T, c->d_scaling,
                                  kListRel, c->d_lrowtot, c->d_lrowoff, c->d_sort_flag, c->d_lpat,
                                  c->d_lx, c->st));
  } else {
    CK(c, launch_list_from_candidates(a, c->cand_n, kListRel, c->d_cand_P, c->d_T64,
                                      c->d_lrowtot, c->d_lcursor, c->d_lrowoff, c->d_lpat,
                                      c->d_lx, c->st));
  }
  c->list_mode = true;
  CK(c, launch_sum_f64(c->d_plogp, N, c->d_stats + 2, c->st));
  CK(c, launch_sum_f64(c->d_lse, N, c->d_stats + 3, c->st));
  c->launches += 7;  // finish, T, count, scan, fill, 2 sums
  return EMC_OK;
}

// The non-zero entries of M [rows][cols] (device, FP32) into s: one warp per
// row counts them, the host scans the counts, a second pass writes each row's
// entries in column order (ballot compaction), so sums over them run in a
// fixed order.  with_aux allocates a second value array of the same length.
static emc_status build_rows(emc_context* c, const float* M, int64_t rows, int64_t cols,
                             SparseRows& s, bool with_aux) {
  if (!s.ptr) TRY(c->alloc(&s.ptr, rows + 1));
  std::vector<int64_t> cnt(rows), ptr(rows + 1, 0);
  int64_t* d_cnt = s.ptr + 1;  // counts land where ptr[1..rows] goes
  CK(c, launch_csr_count(M, rows, cols, d_cnt, c->st));
  CK(c, cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int64_t) * rows, cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  for (int64_t r = 0; r < rows; ++r) ptr[r + 1] = ptr[r] + cnt[r];
  const int64_t nnz = ptr[rows];
  if (nnz + 1 > s.cap || (with_aux && !s.aux)) {
    for (void* q : {(void*)s.idx, (void*)s.val, (void*)s.aux})
      if (q) c->release(q);
    s.idx = nullptr;
    s.val = nullptr;
    s.aux = nullptr;
    s.cap = 0;
    TRY(c->alloc(&s.idx, nnz + 1));
    TRY(c->alloc(&s.val, nnz + 1));
    if (with_aux) TRY(c->alloc(&s.aux, nnz + 1));
    s.cap = nnz + 1;
  }
  CK(c, cudaMemcpyAsync(s.ptr, ptr.data(), sizeof(int64_t) * (rows + 1), cudaMemcpyHostToDevice,
                        c->st));
  CK(c, launch_csr_fill(M, rows, cols, s.ptr, s.idx, s.val, c->st));
  s.nnz = nnz;
  s.valid = true;
  return EMC_OK;
}

// The poisson log-likelihood as a gather over each pattern's photon list:
// the counts' entries by pattern (built once per pattern upload) and log W
// transposed to pixel-major rows so a block of rotations reads one coalesced
// row per photon.
static emc_status sparse_loglik(emc_context* c) {
  const int64_t N = c->N, R = c->R, npa = c->npa;
  if (!c->csr.valid) TRY(build_rows(c, c->d_K, N, npa, c->csr, false));
  const int64_t ldT = (R + 3) / 4 * 4;
  if (!c->d_ST) TRY(c->alloc(&c->d_ST, npa * ldT));
  CK(c, launch_transpose(c->d_S, R, npa, c->d_ST, ldT, c->st));
  SparseLLArgs a{};
  a.row_ptr = c->csr.ptr;
  a.col = c->csr.idx;
  a.val = c->csr.val;
  a.logWT = c->d_ST;
  a.ldT = ldT;
  a.scaling = c->d_scaling;
  a.rowstat = c->d_rowstat;
  a.R = R;
  a.N = N;
  a.LL = c->d_LL;
  a.LL64 = c->d_LL64;
  CK(c, launch_ll_sparse(a, c->st));
  c->launches += 2;
  return EMC_OK;
}

// The slice sums U[r][j] = sum_p P_rp K_pj / phi_p / T_r as a gather over
// each active pixel's non-zero counts: the counts' entries by pixel (built
// once per pattern upload from a transposed copy of K), divided by the
// current scaling, and P transposed to pattern-major rows.
static emc_status sparse_slicesums(emc_context* c) {
  const int64_t N = c->N, R = c->R, npa = c->npa;
  if (!c->csc.valid) {
    float* KT = nullptr;
    TRY(c->alloc(&KT, npa * N));
    CK(c, launch_transpose(c->d_K, N, npa, KT, N, c->st));
    const emc_status s = build_rows(c, KT, npa, N, c->csc, true);
    cudaStreamSynchronize(c->st);
    c->release(KT);
    if (s != EMC_OK) return s;
  }
  const int64_t ldT = (R + 3) / 4 * 4;
  if (!c->d_PT) TRY(c->alloc(&c->d_PT, N * ldT));
  CK(c, launch_transpose(c->d_LL, R, N, c->d_PT, ldT, c->st));
  CK(c, launch_scale_entries(c->csc.val, c->csc.idx, c->d_scaling, c->csc.nnz, c->csc.aux,
                             c->st));
  SparseCmpArgs a{};
  a.col_ptr = c->csc.ptr;
  a.row = c->csc.idx;
  a.val = c->csc.aux;
  a.PT = c->d_PT;
  a.ldT = ldT;
  a.T = c->d_T;
  a.R = R;
  a.npa = npa;
  a.U = c->d_S;
  CK(c, launch_compress_sparse(a, c->st));
  c->launches += 3;
  return EMC_OK;
}

extern "C" {

emc_status emc_maximize(emc_context* c) {
  StageRange range("emc maximize");
  if (!c) return EMC_ERR_ARG;
  if (c->stage != 1) return c->fail(EMC_ERR_STATE, "maximize called before expand");
  const int64_t R = c->R, N = c->N;
  CK(c, cudaMemcpyAsync(c->d_scaling_prev, c->d_scaling, sizeof(float) * N,
                        cudaMemcpyDeviceToDevice, c->st));
  if (!c->mixed && c->tune.maximize_sparse) {
    TRY(sparse_loglik(c));
  } else if (!c->mixed) {
    LLArgs l{};
    l.A = c->d_S;
    l.K = c->d_K;
    l.scaling = c->d_scaling;
    l.rowstat = c->d_rowstat;
    l.R = R;
    l.N = N;
    l.npa = c->npa;
    l.ldA = c->npa;
    l.ldK = c->npa;
    l.ldLL = N;
    l.gauss_inv = gauss_inv(c);
    l.poisson = c->gauss ? 0 : 1;
    l.LL = c->d_LL;
    l.LL64 = c->d_LL64;
    CK(c, launch_ll_fp32(l, c->st));
  }
  if (!c->mixed) {
    c->mark(2);
    int nparts = 0;
    CK(c, launch_softmax_from_f64(c->d_LL64, c->d_LL, R, N, c->d_plogp_part, &nparts,
                                  c->d_lse32, c->st));
    CK(c, launch_sum_f64(c->d_plogp_part, nparts, c->d_stats + 2, c->st));
    CK(c, launch_sum_f64(c->d_lse32, N, c->d_stats + 3, c->st));
    int64_t nden = 0;
    if (c->gauss) {
      CrossArgs x{};
      x.S = c->d_S;
      x.K = c->d_K;
      x.P = c->d_LL;
      x.R = R;
      x.N = N;
      x.npa = c->npa;
      x.ldS = c->npa;
      x.ldK = c->npa;
      x.den_part = c->d_den;
      CK(c, launch_scaling_cross(x, c->st));
      nden = (R + 127) / 128;
    } else {
      CK(c, launch_scaling_rowweighted(c->d_LL, c->d_rowstat, R, N, c->d_den, &nden, c->st));
    }
    CK(c, launch_scaling_finish(c->gauss ? c->d_patsq : c->d_patsum, c->d_den, nden, N,
                                c->d_scaling, c->st));
    CK(c, launch_row_sums(c->d_LL, R, N, c->d_T, c->st));
    c->launches += 8;
  } else if (c->y_rows < R) {
    TRY(chunked_maximize(c));
  } else {
    MaxEpiArgs e = max_args(c);
    if (c->tune.maximize_pair)
      CK(c, launch_maximize_pair_tc(c->tmKh64, c->tmBhi64, c->tmBlo64, c->Npad, c->Rpad, c->Ppad,
                                    e, c->d_status, c->num_sms, c->st, c->tune.maximize_raster));
    else
      CK(c, launch_maximize_tc(c->tmKh, c->tmBhi, c->tmBlo, c->Npad, c->Rpad, c->Ppad, e,
                               c->d_status, c->num_sms, c->st, c->tune.maximize_raster));
    c->mark(2);
    TRY(mixed_resp_pass(c));
    c->launches += 1;  // the maximize contraction
  }
  // the insertion skip test reads Tskip: this context's T_r unless a
  // pattern-sharded caller replaces it by the sum over every shard
  CK(c, cudaMemcpyAsync(c->d_Tskip, c->d_T, sizeof(float) * R, cudaMemcpyDeviceToDevice, c->st));
  c->mark(3);
  c->resp_source = c->mixed && c->y_rows < R ? 3 : 1;
  c->stage = 2;
  return EMC_OK;
}

emc_status emc_compress_insert(emc_context* c) {
  StageRange range("emc compress");
  if (!c) return EMC_ERR_ARG;
  if (c->stage != 2) return c->fail(EMC_ERR_STATE, "compress called before maximize");
  // emc.c:1025-1026 reset, then emc_cuda.cu:292-362 insert, :414-433 normalise
  if (c->det) {
    CK(c, cudaMemsetAsync(c->d_acc64, 0, sizeof(unsigned long long) * 8 * c->M, c->st));
  } else if (!c->mixed) {
    CK(c, cudaMemsetAsync(c->d_model, 0, sizeof(float) * c->M, c->st));
    CK(c, cudaMemsetAsync(c->d_weight, 0, sizeof(float) * c->M, c->st));
  } else {
    CK(c, cudaMemsetAsync(c->d_acc, 0, sizeof(float2) * c->M, c->st));
  }
  if (!c->mixed) {
    if (c->tune.compress_sparse) {
      TRY(sparse_slicesums(c));
    } else {
      CompressArgs a{};
      a.P = c->d_LL;
      a.K = c->d_K;
      a.scaling = c->d_scaling;
      a.T = c->d_T;
      a.R = c->R;
      a.N = c->N;
      a.npa = c->npa;
      a.ldK = c->npa;
      a.ldU = c->npa;
      a.U = c->d_S;  // the averaged slices replace the expanded ones (emc_atomic.cu:96)
      CK(c, launch_compress_fp32(a, c->st));
    }
    InsertArgs in{};
    in.U = c->d_S;
    in.T = c->d_T;
    in.Tskip = c->d_Tskip;
    in.rotw = c->d_rotw;
    in.quat = c->d_quat;
    in.cx = c->d_cx;
    in.cy = c->d_cy;
    in.cz = c->d_cz;
    in.ins = c->d_ins;
    in.R = c->R;
    in.npix = c->npa;
    in.ldU = c->npa;
    in.side = c->cfg.side;
    in.interp = c->cfg.interp;
    in.model = c->d_model;
    in.weight = c->d_weight;
    in.acc64 = c->det ? c->d_acc64 : nullptr;
    CK(c, launch_insert(in, c->st));
    c->launches += 2;
  } else {
    CmpEpiArgs e = cmp_args(c);
    e.acc64 = c->det ? c->d_acc64 : nullptr;
    if (c->list_mode) {
      // responsibility lists x the counts' photon lists (built once per upload)
      if (!c->csr.valid) TRY(build_rows(c, c->d_K, c->N, c->npa, c->csr, false));
      ListCmpArgs la{};
      la.rowoff = c->d_lrowoff;
      la.pat = c->d_lpat;
      la.xv = c->d_lx;
      la.kptr = c->csr.ptr;
      la.kidx = c->csr.idx;
      la.kval = c->csr.val;
      la.e = e;
      la.ordered = c->det ? 1 : 0;
      CK(c, launch_list_compress(la, c->st));
    } else if (c->tune.compress_pair) {
      CK(c, launch_compress_pair_tc(c->tmPhi, c->tmPlo, c->tmKt128, c->Rpad, c->Ppad, c->Npad, e,
                                    c->d_status, c->num_sms, c->st, c->tune.compress_raster));
    } else {
      CK(c, launch_compress_tc(c->tmPhi, c->tmPlo, c->tmKt, c->Rpad, c->Ppad, c->Npad, e,
                               c->d_status, c->num_sms, c->st, c->tune.compress_raster));
    }
    c->launches += 1;
  }
  if (c->det) {
    // the exact sums as the FP32 accumulators the normalisation (and a
    // pattern-sharded caller's all-reduce) read
    if (c->mixed)
      CK(c, launch_fixed_to_pairs(c->d_acc64, c->M, reinterpret_cast<float*>(c->d_acc),
                                  reinterpret_cast<float*>(c->d_acc) + 1, 2, c->st));
    else
      CK(c, launch_fixed_to_pairs(c->d_acc64, c->M, c->d_model, c->d_weight, 1, c->st));
    c->launches += 1;
  }
  c->mark(4);
  c->stage = 3;
  return EMC_OK;
}

emc_status emc_normalize(emc_context* c) {
  StageRange range("emc normalize");
  if (!c) return EMC_ERR_ARG;
  if (c->stage != 3) return c->fail(EMC_ERR_STATE, "normalize called before compress_insert");
  if (!c->mixed)
    CK(c, launch_normalize_model(c->d_model, c->d_weight, c->M, 0, c->d_scratch, c->d_stats,
                                 c->st));
  else
    CK(c, launch_normalize_acc(c->d_acc, c->d_model, c->d_weight, c->M, c->d_scratch,
                               c->d_stats, c->st));
  c->launches += 4;
  c->mark(5);
  c->stage = 0;
  return EMC_OK;
}

emc_status emc_compress(emc_context* c) {
  TRY(emc_compress_insert(c));
  return emc_normalize(c);
}

static emc_status check_status(emc_context* c) {
  TcStatus h{};
  CK(c, cudaMemcpyAsync(&h, c->d_status, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  if (h.code != 0) {
    cudaMemsetAsync(c->d_status, 0, sizeof(TcStatus), c->st);
    cudaStreamSynchronize(c->st);
    return c->fail(EMC_ERR_TIMEOUT, "tensor-core kernel wait %d timed out in block %d", h.where,
                   h.block);
  }
  return EMC_OK;
}

emc_status emc_synchronize(emc_context* c) {
  if (!c) return EMC_ERR_ARG;
  return check_status(c);
}

emc_status emc_wait_probe(emc_context* c, uint32_t limit_us) {
  if (!c || limit_us < 1 || limit_us > 1000000) return EMC_ERR_ARG;
  if (c->stage != 0) return c->fail(EMC_ERR_STATE, "wait probe between iterations");
  TRY(check_status(c));
  CK(c, launch_wait_probe(c->d_status, (uint64_t)limit_us * 1000ull, c->st));
  return check_status(c);
}

emc_status emc_iterate(emc_context* c, emc_iter_stats* stats) {
  TRY(emc_expand(c));
  TRY(emc_maximize(c));
  TRY(emc_compress(c));
  if (stats) {
    TRY(check_status(c));
    double h[4] = {0, 0, 0, 0};
    CK(c, cudaMemcpy(h, c->d_stats, sizeof(h), cudaMemcpyDeviceToHost));
    double T = 0;
    std::vector<float> t(c->R);
    CK(c, cudaMemcpy(t.data(), c->d_T, sizeof(float) * c->R, cudaMemcpyDeviceToHost));
    for (float v : t) T += v;
    stats->model_max = h[1];
    stats->sum_plogp = h[2];
    stats->total_loglik = h[3];
    stats->total_resp = T;
  }
  return EMC_OK;
}

emc_status emc_get_tuning(const emc_context* c, emc_tuning* t) {
  if (!c || !t) return EMC_ERR_ARG;
  *t = c->tune;
  return EMC_OK;
}

emc_status emc_set_tuning(emc_context* c, const emc_tuning* t) {
  if (!c || !t || t->maximize_raster < 1 || t->compress_raster < 1 ||
      (t->maximize_pair != 0 && t->maximize_pair != 1) ||
      (t->compress_pair != 0 && t->compress_pair != 1) ||
      (t->maximize_sparse != 0 && t->maximize_sparse != 1) ||
      (t->compress_sparse != 0 && t->compress_sparse != 1))
    return EMC_ERR_ARG;
  if (t->compress_sparse && c->mixed && c->npa > kListMaxPixels)
    return c->fail(EMC_ERR_UNSUPPORTED, "responsibility lists need at most %lld active pixels",
                   (long long)kListMaxPixels);
  if (t->maximize_sparse && (c->mixed || c->gauss))
    return c->fail(EMC_ERR_UNSUPPORTED, "the photon-list log-likelihood is an FP32 poisson form");
  if (!t->compress_sparse && c->mixed && c->y_rows < c->R)
    return c->fail(EMC_ERR_STATE, "rotation chunks compress from responsibility lists");
  c->tune = *t;
  return EMC_OK;
}

emc_status emc_autotune(emc_context* c, const int32_t* cand, int32_t n, float* ms,
                        emc_tuning* best) {
  if (!c || !cand || n < 1) return EMC_ERR_ARG;
  for (int32_t i = 0; i < n; ++i)
    if (cand[i] < 1) return c->fail(EMC_ERR_ARG, "raster candidates must be >= 1");
  if (!c->have_geom || !c->have_rot || !c->have_pat || !c->have_model)
    return c->fail(EMC_ERR_STATE, "set geometry, rotations, patterns and model first");
  if (c->stage != 0) return c->fail(EMC_ERR_STATE, "autotune between iterations");
  // every trial iterates from the current model and scaling, restored after
  float* save = nullptr;
  CK(c, cudaMalloc(&save, sizeof(float) * (c->M + c->N)));
  auto restore = [&]() -> emc_status {
    CK(c, cudaMemcpyAsync(c->d_model, save, sizeof(float) * c->M, cudaMemcpyDeviceToDevice, c->st));
    CK(c, cudaMemcpyAsync(c->d_scaling, save + c->M, sizeof(float) * c->N,
                          cudaMemcpyDeviceToDevice, c->st));
    return EMC_OK;
  };
  emc_status s = EMC_OK;
  const bool prof_was = c->prof;
  const emc_tuning keep = c->tune;
  emc_tuning win = keep;
  float bmax = 1e30f, bcmp = 1e30f;
  if ((s = c->cuda(cudaMemcpyAsync(save, c->d_model, sizeof(float) * c->M,
                                   cudaMemcpyDeviceToDevice, c->st), "save model")) == EMC_OK &&
      (s = c->cuda(cudaMemcpyAsync(save + c->M, c->d_scaling, sizeof(float) * c->N,
                                   cudaMemcpyDeviceToDevice, c->st), "save scaling")) == EMC_OK &&
      (s = emc_set_profiling(c, 1)) == EMC_OK) {
    // one untimed iteration first (first-launch costs)
    s = emc_iterate(c, nullptr);
    // FP32 contexts: the dense and the photon-list form of each contraction
    // (the maximize's only for poisson); the candidates do not apply
    for (int32_t form = 0; form < 2 && s == EMC_OK && !c->mixed; ++form) {
      c->tune = keep;
      c->tune.maximize_sparse = form && !c->gauss ? 1 : 0;
      c->tune.compress_sparse = form;
      if ((s = restore()) != EMC_OK || (s = emc_iterate(c, nullptr)) != EMC_OK) break;
      float t[5];
      if ((s = c->cuda(cudaEventSynchronize(c->ev[c->cur][5]), "autotune")) != EMC_OK) break;
      for (int k = 0; k < 5; ++k)
        cudaEventElapsedTime(&t[k], c->ev[c->cur][k], c->ev[c->cur][k + 1]);
      if (t[1] < bmax) {
        bmax = t[1];
        win.maximize_sparse = c->tune.maximize_sparse;
      }
      if (t[3] < bcmp) {
        bcmp = t[3];
        win.compress_sparse = c->tune.compress_sparse;
      }
      if (ms) {
        ms[0] = bmax;
        ms[n] = bcmp;
      }
    }
    for (int32_t i = 0; i < n && s == EMC_OK && c->mixed; ++i) {
      float tmax = 1e30f;
      for (int32_t pair = 0; pair < 2 && s == EMC_OK; ++pair) {
        c->tune = emc_tuning{cand[i], cand[i], pair, pair, keep.maximize_sparse,
                             keep.compress_sparse};
        if ((s = restore()) != EMC_OK || (s = emc_iterate(c, nullptr)) != EMC_OK) break;
        float t[5];
        if ((s = c->cuda(cudaEventSynchronize(c->ev[c->cur][5]), "autotune")) != EMC_OK) break;
        for (int k = 0; k < 5; ++k)
          cudaEventElapsedTime(&t[k], c->ev[c->cur][k], c->ev[c->cur][k + 1]);
        tmax = t[1] < tmax ? t[1] : tmax;
        if (t[1] < bmax) {
          bmax = t[1];
          win.maximize_raster = cand[i];
          win.maximize_pair = pair;
        }
        if (t[3] < bcmp) {
          bcmp = t[3];
          win.compress_raster = cand[i];
          win.compress_pair = pair;
        }
        if (ms) ms[n + i] = pair == 0 ? t[3] : (t[3] < ms[n + i] ? t[3] : ms[n + i]);
      }
      if (ms) ms[i] = tmax;
    }
  }
  c->tune = s == EMC_OK ? win : keep;
  const emc_status s2 = restore();
  c->prof = prof_was;
  c->prof_iters = 0;
  cudaStreamSynchronize(c->st);
  cudaFree(save);
  if (s != EMC_OK) return s;
  if (s2 != EMC_OK) return s2;
  if (best) *best = c->tune;
  return EMC_OK;
}

emc_status emc_orientation_stats(emc_context* c, int32_t* best_rot, float* best_resp,
                                 float* avg_resp) {
  if (!c) return EMC_ERR_ARG;
  if (c->resp_source == 0 || c->stage == 1)
    return c->fail(EMC_ERR_STATE, "no responsibilities yet");
  const int64_t N = c->N, R = c->R;
  if (!c->d_best) {
    TRY(c->alloc(&c->d_best, N));
    TRY(c->alloc(&c->d_bestp, N));
  }
  if (c->resp_source == 1) {
    if (!c->mixed) {
      CK(c, launch_col_argmax(c->d_LL, R, N, c->d_best, c->d_bestp, c->st));
    } else {
      RespArgs a{};
      a.N = N;
      a.R = R;
      a.ldY = c->Npad;
      a.poisson = c->gauss ? 0 : 1;
      a.Y = c->d_Y;
      a.scaling = c->d_scaling_prev;
      a.rowstat = c->d_rowstat;
      a.patstat = c->d_patsq;
      a.gauss_inv = gauss_inv(c);
      a.lse = c->d_lse;
      CK(c, launch_resp_argmax(a, c->d_best, c->d_bestp, c->st));
    }
    c->launches += 1;
  } else if (c->resp_source == 3) {
    if (!c->d_cand_key) TRY(c->alloc(&c->d_cand_key, N));
    RespArgs a = resp_args(c);
    a.list_rp = c->d_lcomp_rp;
    a.list_P = c->d_lcomp_P;
    CK(c, launch_cand_argmax(a, c->cand_n, c->d_cand_key, c->d_best, c->d_bestp, c->st));
    c->launches += 3;
  }  // a proposed iteration recorded its best candidates itself
  if (best_rot)
    CK(c, cudaMemcpyAsync(best_rot, c->d_best, sizeof(int32_t) * N, cudaMemcpyDeviceToHost, c->st));
  if (best_resp)
    CK(c, cudaMemcpyAsync(best_resp, c->d_bestp, sizeof(float) * N, cudaMemcpyDeviceToHost, c->st));
  std::vector<float> T;
  if (avg_resp) {
    T.resize(R);
    CK(c, cudaMemcpyAsync(T.data(), c->d_T, sizeof(float) * R, cudaMemcpyDeviceToHost, c->st));
  }
  CK(c, cudaStreamSynchronize(c->st));
  // average responsibility of each rotation over the patterns: T_r / N
  for (int64_t r = 0; r < (avg_resp ? R : 0); ++r) avg_resp[r] = (float)((double)T[r] / (double)N);
  return EMC_OK;
}

emc_status emc_partial_stats(emc_context* c, double* plogp, double* loglik) {
  if (!c) return EMC_ERR_ARG;
  double h[4] = {0, 0, 0, 0};
  CK(c, cudaMemcpyAsync(h, c->d_stats, sizeof(h), cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  if (plogp) *plogp = h[2];
  if (loglik) *loglik = h[3];
  return EMC_OK;
}

emc_status emc_get_model(emc_context* c, float* model) {
  return emc_get_buffer(c, EMC_BUF_MODEL, model, sizeof(float) * (c ? c->M : 0));
}

emc_status emc_get_scaling(emc_context* c, float* scaling) {
  return emc_get_buffer(c, EMC_BUF_SCALING, scaling, sizeof(float) * (c ? c->N : 0));
}

// ---------------------------------------------------------- checkpoint --
// File layout (little-endian): "EMCSTAT1", int32 side, likelihood, interp,
// precision, int64 patterns, rotations, iteration, then float model [side^3],
// weight [side^3], scaling [patterns].  The model and the scaling are the
// whole input of the next iteration (emc.c:989-1084 reads nothing else), so a
// context loaded from the file continues exactly where the saved one stopped.
namespace {
constexpr char kStateMagic[8] = {'E', 'M', 'C', 'S', 'T', 'A', 'T', '1'};
struct StateHeader {
  char magic[8];
  int32_t side, likelihood, interp, precision;
  int64_t n_patterns, n_rotations, iteration;
};
}  // namespace

emc_status emc_save_state(emc_context* c, const char* path, int64_t iteration) {
  if (!c || !path) return EMC_ERR_ARG;
  if (!c->have_model) return c->fail(EMC_ERR_STATE, "no model to save");
  if (c->stage != 0) return c->fail(EMC_ERR_STATE, "save the state between iterations");
  TRY(check_status(c));
  std::vector<float> buf(2 * c->M + c->N);
  CK(c, cudaMemcpyAsync(buf.data(), c->d_model, sizeof(float) * c->M, cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaMemcpyAsync(buf.data() + c->M, c->d_weight, sizeof(float) * c->M,
                        cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaMemcpyAsync(buf.data() + 2 * c->M, c->d_scaling, sizeof(float) * c->N,
                        cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  StateHeader h{};
  std::memcpy(h.magic, kStateMagic, 8);
  h.side = c->cfg.side;
  h.likelihood = c->cfg.likelihood;
  h.interp = c->cfg.interp;
  h.precision = c->cfg.precision;
  h.n_patterns = c->N;
  h.n_rotations = c->R;
  h.iteration = iteration;
  FILE* f = std::fopen(path, "wb");
  if (!f) return c->fail(EMC_ERR_ARG, "cannot open %s for writing", path);
  const bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 &&
                  std::fwrite(buf.data(), sizeof(float), buf.size(), f) == buf.size();
  if (std::fclose(f) != 0 || !ok) return c->fail(EMC_ERR_ARG, "short write to %s", path);
  return EMC_OK;
}

emc_status emc_load_state(emc_context* c, const char* path, int64_t* iteration) {
  if (!c || !path) return EMC_ERR_ARG;
  if (c->stage != 0) return c->fail(EMC_ERR_STATE, "load a state between iterations");
  FILE* f = std::fopen(path, "rb");
  if (!f) return c->fail(EMC_ERR_ARG, "cannot open %s", path);
  StateHeader h{};
  std::vector<float> buf(2 * c->M + c->N);
  const bool ok = std::fread(&h, sizeof(h), 1, f) == 1 &&
                  std::fread(buf.data(), sizeof(float), buf.size(), f) == buf.size() &&
                  std::fgetc(f) == EOF;
  std::fclose(f);
  if (!ok || std::memcmp(h.magic, kStateMagic, 8) != 0)
    return c->fail(EMC_ERR_RANGE, "%s is not a state file of this size", path);
  if (h.side != c->cfg.side || h.n_patterns != c->N || h.n_rotations != c->R)
    return c->fail(EMC_ERR_RANGE,
                   "state of side %d / %lld patterns / %lld rotations does not fit this context",
                   h.side, (long long)h.n_patterns, (long long)h.n_rotations);
  if (count_bad(buf.data(), 2 * c->M + c->N, false))
    return c->fail(EMC_ERR_RANGE, "the state holds NaN or infinite values");
  CK(c, cudaMemcpyAsync(c->d_model, buf.data(), sizeof(float) * c->M, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_weight, buf.data() + c->M, sizeof(float) * c->M,
                        cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_scaling, buf.data() + 2 * c->M, sizeof(float) * c->N,
                        cudaMemcpyHostToDevice, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  c->have_model = true;
  if (iteration) *iteration = h.iteration;
  return EMC_OK;
}

emc_status emc_get_resp_columns(emc_context* c, int64_t n, const int64_t* patterns, float* out) {
  if (!c || n < 1 || !patterns || !out) return EMC_ERR_ARG;
  for (int64_t a = 0; a < n; ++a)
    if (patterns[a] < 0 || patterns[a] >= c->N) return c->fail(EMC_ERR_ARG, "pattern out of range");
  if (c->resp_source == 0 || c->stage == 1) return c->fail(EMC_ERR_STATE, "no responsibilities yet");
  if (c->mixed && c->resp_source == 1 && c->stage != 2 && c->stage != 0)
    return c->fail(EMC_ERR_STATE, "no responsibilities yet");
  TRY(check_status(c));
  const int64_t R = c->R;
  int64_t* d_cols = nullptr;
  float* d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_cols, sizeof(int64_t) * n);
  if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(float) * R * n);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_cols, patterns, sizeof(int64_t) * n, cudaMemcpyHostToDevice, c->st);
  if (e == cudaSuccess && c->resp_source == 2) {
    e = cudaMemsetAsync(d_out, 0, sizeof(float) * R * n, c->st);
    if (e == cudaSuccess) {
      resp_cols_proposed_kernel<<<(unsigned)((n + 7) / 8), 256, 0, c->st>>>(c->last_group, d_cols,
                                                                            n, d_out);
      e = cudaGetLastError();
    }
  } else if (e == cudaSuccess && c->resp_source == 3) {
    // rotation chunks: the candidates' P, 0 elsewhere (every dropped entry is
    // below kListMinP)
    e = cudaMemsetAsync(d_out, 0, sizeof(float) * R * n, c->st);
    if (e == cudaSuccess)
      e = launch_cand_columns(c->d_lcomp_rp, c->d_cand_P, c->cand_n, d_cols, n, d_out, c->st);
  } else if (e == cudaSuccess) {
    const unsigned grid = (unsigned)std::min<int64_t>((R * n + 255) / 256, 8192);
    if (!c->mixed)
      resp_cols_dense_kernel<<<grid, 256, 0, c->st>>>(c->d_LL, nullptr, c->N, 0, nullptr, nullptr,
                                                      nullptr, 0.0, nullptr, R, d_cols, n, d_out);
    else
      resp_cols_dense_kernel<<<grid, 256, 0, c->st>>>(
          nullptr, c->d_Y, c->Npad, c->gauss ? 0 : 1, c->d_scaling_prev, c->d_rowstat, c->d_patsq,
          gauss_inv(c), c->d_lse, R, d_cols, n, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, d_out, sizeof(float) * R * n, cudaMemcpyDeviceToHost, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  cudaFree(d_cols);
  cudaFree(d_out);
  return c->cuda(e, "emc_get_resp_columns");
}

emc_status emc_device_buffer(emc_context* c, emc_buffer which, void** dptr, size_t* bytes) {
  if (!c || !dptr) return EMC_ERR_ARG;
  void* p = nullptr;
  size_t n = 0;
  switch (which) {
    case EMC_BUF_MODEL: p = c->d_model; n = sizeof(float) * c->M; break;
    case EMC_BUF_WEIGHT: p = c->d_weight; n = sizeof(float) * c->M; break;
    case EMC_BUF_SCALING: p = c->d_scaling; n = sizeof(float) * c->N; break;
    case EMC_BUF_TOTALRESP: p = c->d_T; n = sizeof(float) * c->R; break;
    case EMC_BUF_TOTALRESP_ALL: p = c->d_Tskip; n = sizeof(float) * c->R; break;
    case EMC_BUF_ACCUM:
      p = c->mixed ? (void*)c->d_acc : (void*)c->d_model;
      n = sizeof(float) * 2 * c->M;
      break;
    case EMC_BUF_RESP:
      if (c->mixed) return c->fail(EMC_ERR_UNSUPPORTED, "mixed path keeps no FP32 responsibility matrix");
      if (c->resp_source == 2)
        return c->fail(EMC_ERR_STATE, "a proposed iteration's responsibilities are read with "
                                      "emc_get_buffer");
      p = c->d_LL; n = sizeof(float) * c->R * c->N; break;
    case EMC_BUF_SLICES:
      if (c->mixed) return c->fail(EMC_ERR_UNSUPPORTED, "mixed path keeps FP16 hi/lo slices");
      p = c->d_S; n = sizeof(float) * c->R * c->npa; break;
    default: return EMC_ERR_ARG;
  }
  *dptr = p;
  if (bytes) *bytes = n;
  return EMC_OK;
}

emc_status emc_get_buffer(emc_context* c, emc_buffer which, void* host, size_t bytes) {
  if (!c || !host) return EMC_ERR_ARG;
  TRY(check_status(c));
  if (which == EMC_BUF_RESP && c->resp_source == 2) {
    // a proposed iteration: P over each pattern's candidate cells, 0 elsewhere
    const size_t n = (size_t)(c->R * c->N);
    if (bytes != n * sizeof(float)) return c->fail(EMC_ERR_ARG, "buffer size mismatch");
    if (c->stage != 0) return c->fail(EMC_ERR_STATE, "no responsibilities yet");
    float* tmp = nullptr;
    CK(c, cudaMalloc(&tmp, n * sizeof(float)));
    cudaError_t e = launch_proposed_resp(c->last_group, tmp, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(tmp);
    return c->cuda(e, "emc_get_buffer");
  }
  if (c->mixed && (which == EMC_BUF_RESP || which == EMC_BUF_SLICES)) {
    const size_t n = which == EMC_BUF_RESP ? (size_t)(c->R * c->N) : (size_t)(c->R * c->npa);
    if (bytes != n * sizeof(float)) return c->fail(EMC_ERR_ARG, "buffer size mismatch");
    if (which == EMC_BUF_RESP && c->stage != 2 && c->stage != 0)
      return c->fail(EMC_ERR_STATE, "no responsibilities yet");
    float* tmp = nullptr;
    CK(c, cudaMalloc(&tmp, n * sizeof(float)));
    cudaError_t e;
    if (which == EMC_BUF_RESP && c->resp_source == 3) {
      // rotation chunks: the candidates' P, 0 elsewhere (below kListMinP)
      e = cudaMemsetAsync(tmp, 0, n * sizeof(float), c->st);
      if (e == cudaSuccess)
        e = launch_cand_scatter(c->d_lcomp_rp, c->d_cand_P, c->cand_n, c->N, tmp, c->st);
    } else if (which == EMC_BUF_RESP) {
      RespArgs a{};
      a.N = c->N;
      a.R = c->R;
      a.ldY = c->Npad;
      a.poisson = c->gauss ? 0 : 1;
      a.Y = c->d_Y;
      a.scaling = c->d_scaling_prev;
      a.rowstat = c->d_rowstat;
      a.patstat = c->d_patsq;
      a.gauss_inv = gauss_inv(c);
      a.lse = c->d_lse;
      e = launch_resp_export(a, tmp, c->st);
    } else {
      split_sum_kernel<<<dim3(8, (unsigned)(c->R < 65535 ? c->R : 65535)), 256, 0, c->st>>>(
          c->d_Bhi, c->d_Blo, c->R, c->Ppad, c->npa, c->d_rank, tmp);
      e = cudaGetLastError();
      for (int64_t r0 = 65535; r0 < c->R && e == cudaSuccess; r0 += 65535) {
        const int64_t rows = c->R - r0 < 65535 ? c->R - r0 : 65535;
        split_sum_kernel<<<dim3(8, (unsigned)rows), 256, 0, c->st>>>(
            c->d_Bhi + r0 * c->Ppad, c->d_Blo + r0 * c->Ppad, rows, c->Ppad, c->npa, c->d_rank,
            tmp + r0 * c->npa);
        e = cudaGetLastError();
      }
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(tmp);
    return c->cuda(e, "emc_get_buffer");
  }
  void* p = nullptr;
  size_t n = 0;
  TRY(emc_device_buffer(c, which, &p, &n));
  if (bytes != n) return c->fail(EMC_ERR_ARG, "buffer size mismatch (%zu != %zu)", bytes, n);
  CK(c, cudaMemcpyAsync(host, p, n, cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  return EMC_OK;
}


// ----------------------------------------------------- learned proposal --

emc_status emc_set_cells(emc_context* c, const int32_t* cell, int32_t n_cells) {
  if (!c || !cell || n_cells < 1) return EMC_ERR_ARG;
  if (n_cells > 1024) return c->fail(EMC_ERR_RANGE, "at most 1024 cells");
  std::vector<int64_t> beg(n_cells, -1);
  std::vector<int32_t> cnt(n_cells, 0);
  for (int64_t r = 0; r < c->R; ++r) {
    if (cell[r] < 0 || cell[r] >= n_cells) return c->fail(EMC_ERR_ARG, "cell id out of range");
    if (r > 0 && cell[r] < cell[r - 1])
      return c->fail(EMC_ERR_ARG, "rotations must be sorted by cell (cell ids non-decreasing)");
    if (beg[cell[r]] < 0) beg[cell[r]] = r;
    cnt[cell[r]]++;
  }
  for (int32_t k = 0; k < n_cells; ++k)
    if (beg[k] < 0) beg[k] = 0;
  if (!c->d_cell) TRY(c->alloc(&c->d_cell, c->R));
  if (c->n_cells != n_cells) {
    TRY(c->alloc(&c->d_mbeg, n_cells));
    TRY(c->alloc(&c->d_mcnt, n_cells));
    TRY(c->alloc(&c->d_gbeg, n_cells));
    TRY(c->alloc(&c->d_gcnt, n_cells));
    TRY(c->alloc(&c->d_goff, n_cells));
  }
  CK(c, cudaMemcpyAsync(c->d_cell, cell, sizeof(int32_t) * c->R, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_mbeg, beg.data(), sizeof(int64_t) * n_cells, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_mcnt, cnt.data(), sizeof(int32_t) * n_cells, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  c->n_cells = n_cells;
  c->h_mbeg = beg;
  c->h_mcnt = cnt;
  c->max_members = 0;
  for (int32_t k : cnt) c->max_members = k > c->max_members ? k : c->max_members;
  return EMC_OK;
}

emc_status emc_pattern_features(emc_context* c, int32_t in_side, float* x) {
  if (!c || !x) return EMC_ERR_ARG;
  if (!c->have_pat) return c->fail(EMC_ERR_STATE, "patterns are not set");
  if (in_side * 2 != c->cfg.side) return c->fail(EMC_ERR_ARG, "in_side must be side / 2");
  CK(c, launch_features(c->d_K, c->d_pix, c->N, c->npa, c->cfg.side, in_side, x, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  return EMC_OK;
}

}  // extern "C"

// Cell masses (take_log: their logs) of a chunked iteration from its
// candidates, summed in FP64 (a temporary [N][n_cells] accumulator).
static emc_status cand_cells(emc_context* c, float* t, int take_log) {
  const int64_t count = c->N * (int64_t)c->n_cells;
  double* acc = nullptr;
  cudaError_t e = cudaMalloc(&acc, sizeof(double) * count);
  if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, sizeof(double) * count, c->st);
  if (e == cudaSuccess)
    e = launch_cand_cells(c->d_lcomp_rp, c->d_cand_P, c->cand_n, c->d_cell, c->n_cells, acc, c->st);
  if (e == cudaSuccess) e = launch_cells_out(acc, count, take_log, t, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  cudaFree(acc);
  return c->cuda(e, "cell masses of a chunked iteration");
}

extern "C" {

emc_status emc_cell_targets(emc_context* c, float* t) {
  if (!c || !t) return EMC_ERR_ARG;
  if (!c->n_cells) return c->fail(EMC_ERR_STATE, "emc_set_cells first");
  if (c->resp_source == 0 || c->stage == 1)
    return c->fail(EMC_ERR_STATE, "no responsibilities yet");
  if (c->resp_source == 2) {
    CK(c, launch_scatter_targets(c->d_cand, c->d_cmass, c->N, c->cand_m, c->n_cells, t, c->st));
    CK(c, cudaStreamSynchronize(c->st));
    return EMC_OK;
  }
  if (c->resp_source == 3) {
    TRY(cand_cells(c, t, 0));
    CK(c, cudaStreamSynchronize(c->st));
    return EMC_OK;
  }
  TargetArgs a{};
  a.N = c->N;
  a.R = c->R;
  a.n_cells = c->n_cells;
  a.cell = c->d_cell;
  a.mbeg = c->d_mbeg;
  a.mcnt = c->d_mcnt;
  if (!c->mixed) {
    a.P = c->d_LL;
    a.ldP = c->N;
  } else {
    a.Y = c->d_Y;
    a.ldY = c->Npad;
    a.poisson = c->gauss ? 0 : 1;
    a.lse = c->d_lse;
    a.scaling = c->d_scaling_prev;
    a.rowstat = c->d_rowstat;
    a.patstat = c->d_patsq;
    a.gauss_inv = gauss_inv(c);
  }
  a.t = t;
  CK(c, launch_targets(a, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  return EMC_OK;
}

}  // extern "C"


extern "C" {

}  // extern "C"

// Parameters of one proposed iteration.
struct ProposedPlan {
  int32_t m = 1;              // candidate slots per pattern
  float threshold = 0.0f;     // dense fallback when the mean predicted mass is below this
  int32_t audit = 0;          // patterns evaluated against every rotation (0: none)
  float min_captured = 0.0f;  // dense fallback when an audited pattern keeps less than this
};

// Gathers what the dense audit of the sampled patterns needs: their scaling,
// their sum K^2, their pattern index for the FP16 row gather (slots beyond n:
// -1, zero rows), and for FP32 contexts their compact counts.
__global__ void gather_audit_kernel(const int64_t* pat, int n, int nslot, const float* scaling,
                                    const double* patsq, const float* K, int64_t npa,
                                    float* scal_out, double* patsq_out, int32_t* slot_out,
                                    float* K_out) {
  const int a = blockIdx.x;
  if (a >= nslot) return;
  const int64_t p = a < n ? pat[a] : -1;
  if (threadIdx.x == 0) {
    slot_out[a] = (int32_t)p;
    if (a < n) {
      scal_out[a] = scaling[p];
      patsq_out[a] = patsq[p];
    }
  }
  if (K_out && a < n)
    for (int64_t j = threadIdx.x; j < npa; j += blockDim.x) K_out[a * npa + j] = K[p * npa + j];
}

// The dense audit: every rotation's log-likelihood for `audit` sampled
// patterns (the mixed path's maximize contraction on their gathered counts,
// or the FP32 contraction), then the share of each one's responsibility on
// its candidate cells; the result is copied to the host behind ev_audit.
static emc_status run_audit(emc_context* c, int32_t n_aud, int32_t m, float** host_captured) {
  const int64_t R = c->R, N = c->N;
  const int32_t nslot = 128;
  if (!c->d_aud_pat) {
    TRY(c->alloc(&c->d_aud_pat, nslot));
    TRY(c->alloc(&c->d_aud_slot, nslot));
    TRY(c->alloc(&c->d_aud_scal, nslot));
    TRY(c->alloc(&c->d_aud_patsq, nslot));
    TRY(c->alloc(&c->d_aud_cap, nslot));
    if (c->mixed) {
      TRY(c->alloc(&c->d_aud_K16, nslot * c->Ppad, true));
      TRY(c->alloc(&c->d_aud_Y, R * nslot));
      TRY(c->alloc(&c->d_aud_part, c->nrt * nslot));
      if (!tc_encode_2d(&c->tm_aud, c->d_aud_K16, c->Ppad, nslot, 128, kMaximizeBK))
        return c->fail(EMC_ERR_CUDA, "tensor map of the audit counts");
    } else {
      TRY(c->alloc(&c->d_aud_K32, nslot * c->npa));
      TRY(c->alloc(&c->d_aud_LL, R * nslot));
    }
  }
  // an evenly strided sample, shifted every call
  std::vector<int64_t> pat(n_aud);
  const int64_t stride = std::max<int64_t>(1, N / n_aud);
  for (int32_t a = 0; a < n_aud; ++a) pat[a] = (c->audit_round + (int64_t)a * stride) % N;
  c->audit_round = (c->audit_round + 7919) % N;
  int64_t* hp = c->pinned<int64_t>(6, n_aud);
  if (!hp) return c->fail(EMC_ERR_OOM, "pinned host staging");
  std::copy(pat.begin(), pat.end(), hp);
  CK(c, cudaMemcpyAsync(c->d_aud_pat, hp, sizeof(int64_t) * n_aud, cudaMemcpyHostToDevice, c->st));
  gather_audit_kernel<<<nslot, 128, 0, c->st>>>(c->d_aud_pat, n_aud, nslot, c->d_scaling,
                                                c->d_patsq, c->mixed ? nullptr : c->d_K, c->npa,
                                                c->d_aud_scal, c->d_aud_patsq, c->d_aud_slot,
                                                c->mixed ? nullptr : c->d_aud_K32);
  CK(c, cudaGetLastError());
  AuditArgs a{};
  a.R = R;
  a.ld = nslot;
  a.m = m;
  a.poisson = c->gauss ? 0 : 1;
  a.pat = c->d_aud_pat;
  a.cand = c->d_cand;
  a.cell = c->d_cell;
  a.scaling = c->d_aud_scal;
  a.rowstat = c->d_rowstat;
  a.patstat = c->d_aud_patsq;
  a.gauss_inv = gauss_inv(c);
  a.captured = c->d_aud_cap;
  if (c->mixed) {
    CK(c, launch_gather_slots(c->d_Kh, c->Ppad, c->d_aud_slot, nslot, c->d_aud_K16, c->st));
    MaxEpiArgs e{};
    e.N = n_aud;
    e.R = R;
    e.ldY = nslot;
    e.poisson = a.poisson;
    e.scaling = c->d_aud_scal;
    e.rowstat = c->d_rowstat;
    e.patstat = c->d_aud_patsq;
    e.gauss_inv = a.gauss_inv;
    e.Y = c->d_aud_Y;
    e.part = c->d_aud_part;
    CK(c, launch_maximize_tc(c->tm_aud, c->tmBhi, c->tmBlo, nslot, c->Rpad, c->Ppad, e,
                             c->d_status, c->num_sms, c->st, 1));
    a.Y = c->d_aud_Y;
  } else {
    LLArgs l{};
    l.A = c->d_S;
    l.K = c->d_aud_K32;
    l.scaling = c->d_aud_scal;
    l.rowstat = c->d_rowstat;
    l.R = R;
    l.N = n_aud;
    l.npa = c->npa;
    l.ldA = c->npa;
    l.ldK = c->npa;
    l.ldLL = nslot;
    l.gauss_inv = a.gauss_inv;
    l.poisson = a.poisson;
    l.LL64 = c->d_aud_LL;
    CK(c, launch_ll_fp32(l, c->st));
    a.LL64 = c->d_aud_LL;
  }
  CK(c, launch_audit(a, n_aud, c->st));
  float* hc = c->pinned<float>(7, n_aud);
  if (!hc) return c->fail(EMC_ERR_OOM, "pinned host staging");
  CK(c, cudaMemcpyAsync(hc, c->d_aud_cap, sizeof(float) * n_aud, cudaMemcpyDeviceToHost, c->st));
  if (!c->ev_audit) CK(c, cudaEventCreateWithFlags(&c->ev_audit, cudaEventDisableTiming));
  CK(c, cudaEventRecord(c->ev_audit, c->st));
  c->launches += c->mixed ? 4 : 3;  // gather (2), contraction, audit
  *host_captured = hc;
  return EMC_OK;
}

// One proposed iteration: `select` writes the candidate cells (d_cand,
// [N][m]) and their predicted mass (d_mass) on the context stream.
template <class Select>
static emc_status run_proposed(emc_context* c, const ProposedPlan& pl, Select select,
                               emc_proposal_stats* stats) {
  StageRange range("emc proposed iteration");
  const int32_t m = pl.m;
  const int64_t N = c->N, R = c->R, pairs = N * m;
  if (!c->d_mass) {
    TRY(c->alloc(&c->d_mass, N));
    TRY(c->alloc(&c->d_lse_c, N));
    TRY(c->alloc(&c->d_plogp_c, N));
  }
  if (!c->d_best) {
    TRY(c->alloc(&c->d_best, N));
    TRY(c->alloc(&c->d_bestp, N));
  }
  if (!c->d_acc) TRY(c->alloc(&c->d_acc, c->M));
  if (pairs > c->pairs_cap || c->cand_m != m) {
    int64_t cap = c->pairs_cap;
    TRY(grow(c, &c->d_cand, cap, pairs));
    cap = c->pairs_cap;
    TRY(grow(c, &c->d_ppos, cap, pairs));
    cap = c->pairs_cap;
    TRY(grow(c, &c->d_cmass, cap, pairs));
    cap = c->pairs_cap;
    TRY(grow(c, &c->d_lcmass, cap, pairs));
    c->pairs_cap = cap;
    c->cand_m = m;
  }
  if (c->stage != 0) return c->fail(EMC_ERR_STATE, "proposed iteration between stages");
  // candidate cells of every pattern and the proposal's mass on them; their
  // copy to the host is waited for while the expansion runs behind it
  CK(c, select());
  int32_t* cand = c->pinned<int32_t>(0, pairs);
  float* mass = c->pinned<float>(1, N);
  if (!cand || !mass) return c->fail(EMC_ERR_OOM, "pinned host staging");
  CK(c, cudaMemcpyAsync(cand, c->d_cand, sizeof(int32_t) * pairs, cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaMemcpyAsync(mass, c->d_mass, sizeof(float) * N, cudaMemcpyDeviceToHost, c->st));
  if (!c->ev_sel) CK(c, cudaEventCreateWithFlags(&c->ev_sel, cudaEventDisableTiming));
  CK(c, cudaEventRecord(c->ev_sel, c->st));
  TRY(emc_expand(c));
  if (!c->mixed && c->gauss)  // the grouped gaussian LL uses the expanded form: sum_j S_rj^2
    CK(c, launch_pattern_stats(c->d_S, nullptr, R, c->npa, c->npa, 1, c->d_rowstat, c->st));
  float* captured = nullptr;
  const int32_t n_aud = (int32_t)std::min<int64_t>(pl.audit, std::min<int64_t>(N, 128));
  if (n_aud > 0) TRY(run_audit(c, n_aud, m, &captured));
  CK(c, cudaEventSynchronize(c->ev_sel));
  double msum = 0.0, mmin = 1e300;
  for (int64_t p = 0; p < N; ++p) {
    msum += mass[p];
    mmin = mass[p] < mmin ? mass[p] : mmin;
  }
  emc_proposal_stats st{};
  st.mean_mass = msum / (double)N;
  st.min_mass = mmin;
  auto dense_instead = [&]() -> emc_status {
    TRY(emc_maximize(c));
    TRY(emc_compress(c));
    st.fallback = 1;
    st.pairs = 0;
    st.evaluations = N * R;
    if (stats) *stats = st;
    return EMC_OK;
  };
  // the proposal is not confident enough: the dense iteration runs instead
  if (st.mean_mass < pl.threshold) return dense_instead();
  // Group the (pattern, cell) pairs by cell (stable counting sort on the
  // host).  Pairs live in slots: cell c owns slots gbeg[c] .. gbeg[c]+gcnt[c]-1,
  // its first slot a multiple of 8; the slots between cells are padding
  // (pattern -1).
  const int n_cells = c->n_cells;
  std::vector<int32_t> gcnt(n_cells, 0);
  int64_t npairs = 0;
  for (int64_t p = 0; p < N; ++p)
    for (int32_t i = 0; i < m; ++i) {
      const int32_t k = cand[p * m + i];
      if (k < 0) {
        if (i == 0) return c->fail(EMC_ERR_ARG, "cell probabilities must be finite");
        break;
      }
      if (k >= n_cells) return c->fail(EMC_ERR_ARG, "cell index out of range");
      gcnt[k]++;
      npairs++;
    }
  std::vector<int64_t> gbeg(n_cells), goff(n_cells), fill(n_cells);
  int64_t S = 0, off = 0, evals = 0, kw = 0;
  for (int32_t k = 0; k < n_cells; ++k) {
    gbeg[k] = S;
    fill[k] = S;
    S += (gcnt[k] + 7) / 8 * 8;
    goff[k] = off;
    off += (int64_t)gcnt[k] * c->h_mcnt[k];
    evals += (int64_t)gcnt[k] * c->h_mcnt[k];
    kw = std::max<int64_t>(kw, (gcnt[k] + 63) / 64 * 64);
  }
  int32_t* gpair = c->pinned<int32_t>(2, S);
  int64_t* ppos = c->pinned<int64_t>(3, pairs);
  if (!gpair || !ppos) return c->fail(EMC_ERR_OOM, "pinned host staging");
  std::fill(gpair, gpair + S, -1);
  std::fill(ppos, ppos + pairs, (int64_t)-1);
  for (int64_t p = 0; p < N; ++p)
    for (int32_t i = 0; i < m; ++i) {
      const int32_t k = cand[p * m + i];
      if (k < 0) break;
      const int64_t q = fill[k]++;
      gpair[q] = (int32_t)p;
      ppos[p * m + i] = q;
    }
  // tcgen05 grouped contractions: mixed precision, cells of at most 256 rotations
  const bool tc = c->mixed && c->max_members <= 256 && S > 0 && (S + 31) / 32 <= 65535;
  TRY(grow(c, &c->d_gpair, c->slots_cap, S));
  CK(c, cudaMemcpyAsync(c->d_gpair, gpair, sizeof(int32_t) * S, cudaMemcpyHostToDevice, c->st));
  if (tc) {
    // the slot rows change no state, so they go ahead of the audit's verdict
    // and keep the GPU busy while the host waits for it
    TRY(grow(c, &c->d_Kg, c->kg_cap, S * c->Ppad));
    if (slot_rows_fit(c->Ppad)) {
      // the slot rows from the photon lists (writes the rows, reads the lists)
      if (!c->csr.valid) TRY(build_rows(c, c->d_K, c->N, c->npa, c->csr, false));
      CK(c, launch_slot_rows(c->csr.ptr, c->csr.idx, c->csr.val, c->Ppad, c->d_gpair, S, c->d_Kg,
                             c->st));
    } else {
      CK(c, launch_gather_slots(c->d_Kh, c->Ppad, c->d_gpair, S, c->d_Kg, c->st));
    }
  }
  // the audited patterns' captured responsibility decides between the
  // grouped stages and the dense iteration
  if (n_aud > 0) {
    CK(c, cudaEventSynchronize(c->ev_audit));
    double csum = 0.0, cmin = 1e300;
    for (int32_t a = 0; a < n_aud; ++a) {
      csum += captured[a];
      cmin = captured[a] < cmin ? captured[a] : cmin;
    }
    st.audited = n_aud;
    st.audit_mean_captured = csum / n_aud;
    st.audit_min_captured = cmin;
    if (cmin < pl.min_captured) return dense_instead();
  }
  const int64_t MM = tc ? 256 : c->max_members;
  TRY(grow(c, &c->d_Yc, c->yc_cap, S * MM));
  // compress from responsibility lists (as the dense mixed iteration does);
  // the grouped compresses read the per-cell operand Pt instead
  const bool lists = tc && c->tune.compress_sparse && c->npa <= kListMaxPixels;
  if (!lists) TRY(grow(c, &c->d_Pt, c->pt_cap, evals));
  std::vector<int4> mt, ct;
  int64_t n_gmt = 0, n_gct = 0;
  TileDesc *gmt = nullptr, *gct = nullptr;
  // the grouped maximize on SM pairs (256-slot tiles) where the dense one is
  const bool gpair_form = tc && c->tune.maximize_pair;
  const int32_t gm_rows = gpair_form ? 256 : 128;
  if (tc) {
    const int64_t ptiles = (c->npa + 255) / 256;
    for (int32_t k = 0; k < n_cells; ++k)
      if (gcnt[k] > 0) {
        n_gmt += (gcnt[k] + gm_rows - 1) / gm_rows;
        n_gct += (int64_t)((c->h_mcnt[k] + 127) / 128) * ptiles;
      }
    gmt = c->pinned<TileDesc>(4, n_gmt);
    gct = c->pinned<TileDesc>(5, n_gct);
    if (!gmt || !gct) return c->fail(EMC_ERR_OOM, "pinned host staging");
    int64_t im = 0, ic = 0;
    for (int32_t k = 0; k < n_cells; ++k) {
      if (gcnt[k] == 0) continue;
      for (int32_t q0 = 0; q0 < gcnt[k]; q0 += gm_rows)
        gmt[im++] = TileDesc{(int32_t)(gbeg[k] + q0), 0, (int32_t)c->h_mbeg[k], 0,
                             (int32_t)(c->Ppad / (gpair_form ? kPairBoxK : kMaximizeBK)), k, q0,
                             0};
      for (int32_t r0 = 0; r0 < c->h_mcnt[k]; r0 += 128)
        for (int64_t nt = 0; nt < ptiles; ++nt)
          gct[ic++] = TileDesc{(int32_t)(c->h_mbeg[k] + r0), 0, (int32_t)(nt * 256),
                               (int32_t)gbeg[k], (gcnt[k] + 63) / 64, k, r0, 0};
    }
    TRY(grow(c, &c->d_gmt, c->gmt_cap, n_gmt));
    TRY(grow(c, &c->d_gct, c->gct_cap, n_gct));
    if (!lists && kw > c->a_ld) {
      for (__half** q : {&c->d_Ahi, &c->d_Alo})
        if (*q) {
          c->release(*q);
          *q = nullptr;
        }
      c->a_ld = 0;
      const int64_t ld = (kw + kw / 4 + 63) / 64 * 64;
      TRY(c->alloc(&c->d_Ahi, R * ld));
      TRY(c->alloc(&c->d_Alo, R * ld));
      c->a_ld = ld;
    }
    CK(c, cudaMemcpyAsync(c->d_gmt, gmt, sizeof(TileDesc) * n_gmt, cudaMemcpyHostToDevice, c->st));
    CK(c, cudaMemcpyAsync(c->d_gct, gct, sizeof(TileDesc) * n_gct, cudaMemcpyHostToDevice, c->st));
  } else {
    // CUDA-core grouped contractions: tile lists over the selected cells
    for (int32_t k = 0; k < n_cells; ++k) {
      if (gcnt[k] == 0) continue;
      for (int32_t r0 = 0; r0 < c->h_mcnt[k]; r0 += TM) {
        ct.push_back(make_int4(k, r0, 0, 0));
        for (int32_t q0 = 0; q0 < gcnt[k]; q0 += TN) mt.push_back(make_int4(k, r0, q0, 0));
      }
    }
    TRY(grow(c, &c->d_mtiles, c->mtiles_cap, (int64_t)mt.size()));
    TRY(grow(c, &c->d_ctiles, c->ctiles_cap, (int64_t)ct.size()));
    CK(c, cudaMemcpyAsync(c->d_mtiles, mt.data(), sizeof(int4) * mt.size(), cudaMemcpyHostToDevice, c->st));
    CK(c, cudaMemcpyAsync(c->d_ctiles, ct.data(), sizeof(int4) * ct.size(), cudaMemcpyHostToDevice, c->st));
  }
  CK(c, cudaMemcpyAsync(c->d_ppos, ppos, sizeof(int64_t) * pairs, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_gbeg, gbeg.data(), sizeof(int64_t) * n_cells, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_gcnt, gcnt.data(), sizeof(int32_t) * n_cells, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_goff, goff.data(), sizeof(int64_t) * n_cells, cudaMemcpyHostToDevice, c->st));
  CK(c, cudaMemcpyAsync(c->d_scaling_prev, c->d_scaling, sizeof(float) * N, cudaMemcpyDeviceToDevice, c->st));
  CK(c, cudaMemsetAsync(c->d_T, 0, sizeof(float) * R, c->st));
  GroupArgs g{};
  g.N = N;
  g.R = R;
  g.npa = c->npa;
  g.MM = MM;
  g.n_cells = n_cells;
  g.m = m;
  g.poisson = c->gauss ? 0 : 1;
  g.mbeg = c->d_mbeg;
  g.mcnt = c->d_mcnt;
  g.gbeg = c->d_gbeg;
  g.gcnt = c->d_gcnt;
  g.gpair = c->d_gpair;
  g.ppos = c->d_ppos;
  g.cand = c->d_cand;
  g.goff = c->d_goff;
  if (!c->mixed) {
    g.S = c->d_S;
    g.ldS = c->npa;
  } else {
    g.hi = c->d_Bhi;
    g.lo = c->d_Blo;
    g.ldS = c->Ppad;
  }
  g.K = c->d_K;
  g.scaling = c->d_scaling_prev;
  g.rowstat = c->d_rowstat;
  g.patstat = c->d_patsq;
  g.patsum = c->d_patsum;
  g.gauss_inv = gauss_inv(c);
  g.Y = c->d_Yc;
  g.Pt = lists ? nullptr : c->d_Pt;
  g.T = c->d_T;
  g.lse = c->d_lse_c;
  g.plogp = c->d_plogp_c;
  g.new_scaling = c->d_scaling;
  g.cmass = c->d_cmass;
  g.lcmass = c->d_lcmass;
  g.best_rot = c->d_best;
  g.best_p = c->d_bestp;
  g.mtiles = c->d_mtiles;
  g.ctiles = c->d_ctiles;
  g.rotw = c->d_rotw;
  g.quat = c->d_quat;
  g.cx = c->d_cx;
  g.cy = c->d_cy;
  g.cz = c->d_cz;
  g.ins = c->d_ins;
  g.side = c->cfg.side;
  g.interp = c->cfg.interp;
  g.acc = c->d_acc;
  int launches = 0;
  if (tc) {
    CUtensorMap tmKg, tmKg64, tmAhi, tmAlo;
    if (!tc_encode_2d(&tmKg, c->d_Kg, c->Ppad, S, 128, gpair_form ? kPairBoxK : kMaximizeBK))
      return c->fail(EMC_ERR_CUDA, "tensor map encoding failed");
    if (!lists &&
        (!tc_encode_2d(&tmKg64, c->d_Kg, c->Ppad, S, kCompressBK, 64) ||
         !tc_encode_2d_strided(&tmAhi, c->d_Ahi, c->a_ld, R, c->a_ld, 128, kCompressBK) ||
         !tc_encode_2d_strided(&tmAlo, c->d_Alo, c->a_ld, R, c->a_ld, 128, kCompressBK)))
      return c->fail(EMC_ERR_CUDA, "tensor map encoding failed");
    c->mark(1);
    GMaxEpiArgs ge{};
    ge.tiles = c->d_gmt;
    ge.mcnt = c->d_mcnt;
    ge.gcnt = c->d_gcnt;
    ge.gpair = c->d_gpair;
    ge.poisson = g.poisson;
    ge.scaling = c->d_scaling_prev;
    ge.rowstat = c->d_rowstat;
    ge.Y = c->d_Yc;
    ge.ldY = MM;
    if (gpair_form)
      CK(c, launch_group_maximize_pair_tc(tmKg, c->tmBhi64, c->tmBlo64, n_gmt, ge, c->d_status,
                                          c->num_sms, c->st));
    else
      CK(c, launch_group_maximize_tc(tmKg, c->tmBhi, c->tmBlo, n_gmt, ge, c->d_status,
                                     c->num_sms, c->st));
    c->mark(2);
    CK(c, launch_group_softmax(g, c->st));
    if (lists) {
      if (!c->d_lrowoff) {
        TRY(c->alloc(&c->d_lrowtot, R));
        TRY(c->alloc(&c->d_lrowoff, R + 1));
      }
      if (!c->d_lcursor) TRY(c->alloc(&c->d_lcursor, R));
      // a list entry is an evaluated (rotation, pattern) pair: `evals` bounds
      // their number, so the lists need no count from the device
      TRY(grow(c, &c->d_lpat, c->lcap, evals + 1));
      int64_t cap = c->lcap_x;
      TRY(grow(c, &c->d_lx, cap, evals + 1));
      c->lcap_x = cap;
      CK(c, launch_group_list_count(g, kListRel, c->d_lrowtot, c->st));
      CK(c, launch_list_rowscan(c->d_lrowtot, R, c->d_lrowoff, c->st));
      CK(c, launch_group_list_fill(g, kListRel, c->d_lcursor, c->d_lrowoff, c->d_lpat, c->d_lx,
                                   c->st));
      if (!c->csr.valid) TRY(build_rows(c, c->d_K, c->N, c->npa, c->csr, false));
      c->mark(3);
      CK(c, cudaMemsetAsync(c->d_acc, 0, sizeof(float2) * c->M, c->st));
      ListCmpArgs la{};
      la.rowoff = c->d_lrowoff;
      la.pat = c->d_lpat;
      la.xv = c->d_lx;
      la.kptr = c->csr.ptr;
      la.kidx = c->csr.idx;
      la.kval = c->csr.val;
      la.e = cmp_args(c);
      la.e.Tskip = nullptr;  // the proposed iteration's own T_r
      CK(c, launch_list_compress(la, c->st));
      launches = 7;  // row build, contraction, softmax, count + scan, fill, compress
    } else {
    CK(c, launch_p_split(g, c->d_cell, R, c->d_T, c->a_ld, c->d_Ahi, c->d_Alo, c->st));
    c->mark(3);
    CK(c, cudaMemsetAsync(c->d_acc, 0, sizeof(float2) * c->M, c->st));
    GCmpEpiArgs ce{};
    ce.tiles = c->d_gct;
    ce.mcnt = c->d_mcnt;
    ce.npa = c->npa;
    ce.side = c->cfg.side;
    ce.interp = c->cfg.interp;
    ce.quat = c->d_quat;
    ce.rotw = c->d_rotw;
    ce.T = c->d_T;
    ce.cx = c->d_cx;
    ce.cy = c->d_cy;
    ce.cz = c->d_cz;
    ce.ins = c->d_ins;
    ce.acc = c->d_acc;
    CK(c, launch_group_compress_tc(tmAhi, tmAlo, tmKg64, n_gct, ce, c->d_status,
                                   c->num_sms, c->st));
    launches = 6;  // gather (2), contraction, softmax, split, contraction
    }
  } else {
    c->mark(1);
    CK(c, launch_group_maximize(g, (int64_t)mt.size(), c->st));
    c->mark(2);
    c->mark(3);
    CK(c, cudaMemsetAsync(c->d_acc, 0, sizeof(float2) * c->M, c->st));
    CK(c, launch_group_compress(g, (int64_t)ct.size(), c->st));
    launches = 3;  // contraction, softmax, contraction
  }
  c->resp_source = 2;
  c->last_group = g;
  c->mark(4);
  CK(c, launch_normalize_acc(c->d_acc, c->d_model, c->d_weight, c->M, c->d_scratch, c->d_stats,
                             c->st));
  CK(c, launch_sum_f64(c->d_plogp_c, N, c->d_stats + 2, c->st));
  CK(c, launch_sum_f64(c->d_lse_c, N, c->d_stats + 3, c->st));
  c->mark(5);
  // select, the grouped stages, normalise (4), two sums
  c->launches += 1 + launches + 6 + ((!c->mixed && c->gauss) ? 1 : 0);
  c->stage = 0;
  TRY(check_status(c));
  double h[4];
  CK(c, cudaMemcpy(h, c->d_stats, sizeof(h), cudaMemcpyDeviceToHost));
  st.sum_plogp = h[2];
  st.total_loglik = h[3];
  st.pairs = npairs;
  st.evaluations = evals;
  st.fallback = 0;
  if (stats) *stats = st;
  return EMC_OK;
}

extern "C" {

emc_status emc_iterate_proposed(emc_context* c, const float* probs, const float* keep,
                                int32_t min_m, int32_t m, float mass_target, float keep_mass,
                                float threshold, emc_proposal_stats* stats) {
  if (!c || !probs || m < 1 || min_m < 1 || min_m > m) return EMC_ERR_ARG;
  if (!c->n_cells) return c->fail(EMC_ERR_STATE, "emc_set_cells first");
  if (m > c->n_cells) return c->fail(EMC_ERR_ARG, "more cells per pattern than cells");
  if (c->det) return c->fail(EMC_ERR_UNSUPPORTED, "deterministic insertion is a dense-iteration mode");
  ProposedPlan pl;
  pl.m = m;
  pl.threshold = threshold;
  return run_proposed(c, pl, [&]() {
    return launch_select(probs, keep, c->N, c->n_cells, min_m, m, mass_target, keep_mass,
                         c->d_cand, c->d_mass, c->st);
  }, stats);
}

emc_status emc_iterate_topk(emc_context* c, const float* probs, const float* log_keep,
                            const emc_topk_config* cfg, emc_proposal_stats* stats) {
  if (!c || !cfg || (!probs && !log_keep) || cfg->top_k < 1 || cfg->max_cells < 1 ||
      cfg->audit_patterns < 0 || cfg->audit_patterns > 128 || !(cfg->min_captured <= 1.0f) ||
      !(cfg->keep_tail >= 0.0f && cfg->keep_tail < 1.0f))
    return EMC_ERR_ARG;
  if (!c->n_cells) return c->fail(EMC_ERR_STATE, "emc_set_cells first");
  if (c->det) return c->fail(EMC_ERR_UNSUPPORTED, "deterministic insertion is a dense-iteration mode");
  const int32_t m = std::min<int32_t>(cfg->max_cells, c->n_cells);
  ProposedPlan pl;
  pl.m = m;
  pl.threshold = 0.0f;
  pl.audit = cfg->audit_patterns;
  pl.min_captured = cfg->min_captured;
  return run_proposed(c, pl, [&]() {
    return launch_select_topk(probs, log_keep, c->d_mcnt, c->N, c->n_cells, cfg->top_k, m,
                              cfg->mass_target, cfg->keep_tail, c->d_cand, c->d_mass, c->st);
  }, stats);
}

emc_status emc_cell_log_mass(emc_context* c, float* t) {
  if (!c || !t) return EMC_ERR_ARG;
  if (!c->n_cells) return c->fail(EMC_ERR_STATE, "emc_set_cells first");
  if (c->resp_source == 0 || c->stage == 1)
    return c->fail(EMC_ERR_STATE, "no responsibilities yet");
  if (c->resp_source == 2) {
    CK(c, launch_scatter_log_targets(c->d_cand, c->d_lcmass, c->N, c->cand_m, c->n_cells, t,
                                     c->st));
  } else if (c->resp_source == 3) {
    TRY(cand_cells(c, t, 1));
  } else {
    TargetArgs a{};
    a.N = c->N;
    a.R = c->R;
    a.n_cells = c->n_cells;
    a.cell = c->d_cell;
    a.mbeg = c->d_mbeg;
    a.mcnt = c->d_mcnt;
    if (!c->mixed) {
      a.L64 = c->d_LL64;
      a.ldP = c->N;
      a.lse = c->d_lse32;
    } else {
      a.Y = c->d_Y;
      a.ldY = c->Npad;
      a.poisson = c->gauss ? 0 : 1;
      a.lse = c->d_lse;
      a.scaling = c->d_scaling_prev;
      a.rowstat = c->d_rowstat;
      a.patstat = c->d_patsq;
      a.gauss_inv = gauss_inv(c);
    }
    a.t = t;
    CK(c, launch_log_targets(a, c->st));
  }
  CK(c, cudaStreamSynchronize(c->st));
  return EMC_OK;
}

}  // extern "C"

// ------------------------------------------------ several datasets at once --
// One iteration of several contexts with one persistent launch per
// contraction (a tile list over all datasets), the per-dataset stages in
// between on one shared stream, and optionally the whole iteration captured
// into a CUDA graph.

struct emc_batch {
  std::vector<emc_context*> ctx;
  std::vector<cudaStream_t> own;  // the contexts' own streams, given back by destroy
  cudaStream_t st = nullptr;
  TileDesc *d_mt = nullptr, *d_ct = nullptr;
  int64_t n_mt = 0, n_ct = 0;
  bool pair = false;      // the batched maximize on SM pairs
  bool cmp_pair = false;  // the batched compress on SM pairs
  std::vector<char> alone;  // datasets that keep their own contraction launches
  std::vector<char> lists;  // datasets whose compress reads responsibility lists
  std::vector<int64_t> per_iter;  // each dataset's launches in one captured iteration
  MaxEpiArgs* d_max = nullptr;  // per-dataset epilogue arguments (fixed per context)
  CmpEpiArgs* d_cmp = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::string err;
  emc_status fail(emc_status s, const std::string& m) {
    err = m;
    return s;
  }
  emc_status cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return EMC_OK;
    return fail(e == cudaErrorMemoryAllocation ? EMC_ERR_OOM : EMC_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
  }
};

#define BCK(b, x)                                     \
  do {                                                \
    emc_status _s = (b)->cuda((x), #x);               \
    if (_s != EMC_OK) return _s;                      \
  } while (0)
#define BTRY(b, c, x)                                 \
  do {                                                \
    emc_status _s = (x);                              \
    if (_s != EMC_OK) return (b)->fail(_s, (c)->err); \
  } while (0)

// Dataset i's stages of a batched iteration that are not shared launches.
// The maximize contraction of a dataset with its own launches.
static emc_status batch_own_maximize(emc_batch* b, int i) {
  emc_context* c = b->ctx[i];
  const MaxEpiArgs e = max_args(c);
  if (c->tune.maximize_pair)
    BCK(b, launch_maximize_pair_tc(c->tmKh64, c->tmBhi64, c->tmBlo64, c->Npad, c->Rpad, c->Ppad, e,
                                   c->d_status, c->num_sms, b->st, c->tune.maximize_raster));
  else
    BCK(b, launch_maximize_tc(c->tmKh, c->tmBhi, c->tmBlo, c->Npad, c->Rpad, c->Ppad, e,
                              c->d_status, c->num_sms, b->st, c->tune.maximize_raster));
  c->launches += 1;
  return EMC_OK;
}

// The responsibility pass (lists gated on their device-side count, or the
// dense compress operand) and the compress's starting state.
static emc_status batch_resp(emc_batch* b, int i) {
  emc_context* c = b->ctx[i];
  BTRY(b, c, b->lists[i] ? gated_list_pass(c) : mixed_resp_pass(c, false));
  BCK(b, cudaMemcpyAsync(c->d_Tskip, c->d_T, sizeof(float) * c->R, cudaMemcpyDeviceToDevice,
                         b->st));
  c->resp_source = 1;
  c->stage = 2;
  BCK(b, cudaMemsetAsync(c->d_acc, 0, sizeof(float2) * c->M, b->st));
  return EMC_OK;
}

// The compress of a dataset outside the batched compress: from its lists
// when they fit, else (gated on the same count) its dense contraction; or,
// without lists, its dense contraction.
static emc_status batch_own_compress(emc_batch* b, int i) {
  emc_context* c = b->ctx[i];
  CmpEpiArgs e = cmp_args(c);
  if (b->lists[i]) {
    if (!c->csr.valid) BTRY(b, c, build_rows(c, c->d_K, c->N, c->npa, c->csr, false));
    ListCmpArgs la{};
    la.rowoff = c->d_lrowoff;
    la.pat = c->d_lpat;
    la.xv = c->d_lx;
    la.kptr = c->csr.ptr;
    la.kidx = c->csr.idx;
    la.kval = c->csr.val;
    la.e = e;
    la.gate_count = c->d_lcount;
    la.gate_cap = c->lcomp_cap;
    BCK(b, launch_list_compress(la, b->st));
    e.gate_count = c->d_lcount;
    e.gate_cap = c->lcomp_cap;
    c->launches += 1;
  }
  if (c->tune.compress_pair)
    BCK(b, launch_compress_pair_tc(c->tmPhi, c->tmPlo, c->tmKt128, c->Rpad, c->Ppad, c->Npad, e,
                                   c->d_status, c->num_sms, b->st, c->tune.compress_raster));
  else
    BCK(b, launch_compress_tc(c->tmPhi, c->tmPlo, c->tmKt, c->Rpad, c->Ppad, c->Npad, e,
                              c->d_status, c->num_sms, b->st, c->tune.compress_raster));
  c->launches += 1;
  return EMC_OK;
}

extern "C" {

emc_status emc_batch_destroy(emc_batch* b) {
  if (!b) return EMC_OK;
  if (b->st) cudaStreamSynchronize(b->st);
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    b->ctx[i]->st = b->own[i];
    b->ctx[i]->batched = false;
  }
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_mt) cudaFree(b->d_mt);
  if (b->d_ct) cudaFree(b->d_ct);
  if (b->d_max) cudaFree(b->d_max);
  if (b->d_cmp) cudaFree(b->d_cmp);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return EMC_OK;
}

emc_status emc_batch_create(emc_context* const* ctxs, int32_t n, emc_batch** out) {
  if (!ctxs || !out || n < 1 || n > kMaxBatch) return EMC_ERR_ARG;
  *out = nullptr;
  const int dev = ctxs[0]->cfg.device;
  for (int32_t i = 0; i < n; ++i) {
    emc_context* c = ctxs[i];
    if (!c || !c->mixed || c->cfg.device != dev) return EMC_ERR_ARG;
    if (!c->have_geom || !c->have_rot || !c->have_pat || !c->have_model || c->stage != 0 ||
        c->batched)
      return EMC_ERR_STATE;
    // the batched contractions read every rotation's Y and P' and insert
    // with FP32 atomics
    if (c->y_rows < c->R || c->det) return EMC_ERR_UNSUPPORTED;
    for (int32_t k = 0; k < i; ++k)
      if (ctxs[k] == c) return EMC_ERR_ARG;
  }
  emc_batch* b = new emc_batch();
  if (cudaSetDevice(dev) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess) {
    emc_batch_destroy(b);
    return EMC_ERR_CUDA;
  }
  for (int32_t i = 0; i < n; ++i) {
    cudaStreamSynchronize(ctxs[i]->st);
    b->ctx.push_back(ctxs[i]);
    b->own.push_back(ctxs[i]->st);
    ctxs[i]->st = b->st;  // every stage of every dataset on the batch's stream
    ctxs[i]->batched = true;
  }
  // A dataset whose own maximize fills the persistent grid for
  // kAloneWaves waves gains nothing from sharing it: it keeps its own
  // contraction launches (its tuned form and tile order) inside the batch's
  // iteration and graph, and the batched launches cover the others.
  // Datasets with responsibility lists compress from them (gated_list_pass),
  // with the dense contraction of their own as the gated fallback; the
  // batched compress takes the others.
  for (int32_t i = 0; i < n; ++i) {
    emc_context* c = ctxs[i];
    b->lists.push_back(c->tune.compress_sparse && c->npa <= kListMaxPixels ? 1 : 0);
    if (b->lists.back()) {
      const emc_status ls = batch_lists_ready(
          c, c->cand_cap_min > 0 ? c->cand_cap_min : std::max<int64_t>(64 * c->N, 1 << 20));
      if (ls != EMC_OK) {
        b->err = c->err;
        emc_batch_destroy(b);
        return ls;
      }
    }
  }
  std::vector<int32_t> order;
  for (int32_t i = 0; i < n; ++i) {
    const emc_context* c = ctxs[i];
    const bool pr = c->tune.maximize_pair;
    const int64_t tiles = pr ? ((c->Npad + 255) / 256) * (c->Rpad / 256)
                             : (c->Npad / 128) * (c->Rpad / 256);
    const int64_t wave = pr ? c->num_sms / 2 : c->num_sms;
    b->alone.push_back(tiles >= kAloneWaves * wave ? 1 : 0);
    if (!b->alone.back()) order.push_back(i);
  }
  // Tile lists, the costliest tiles first (a tile's time grows with its K
  // extent), each dataset's tiles in the order of its own launch.
  std::vector<TileDesc> mt, ct;
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t x, int32_t y) { return ctxs[x]->Ppad > ctxs[y]->Ppad; });
  // the order of the single-dataset launch (tile_mn in kernels_tc.cu): the
  // inner index fastest, in bands of `raster` outer tiles
  auto banded = [](int64_t inner, int64_t outer, int64_t raster, auto&& emit) {
    raster = raster < 1 ? 1 : raster;
    for (int64_t o0 = 0; o0 < outer; o0 += raster) {
      const int64_t g = outer - o0 < raster ? outer - o0 : raster;
      for (int64_t w = 0; w < g * inner; ++w) emit(w / g, o0 + w % g);
    }
  };
  // one form for the batched maximize: SM pairs when the datasets that chose
  // them on their own hold most of the work
  double work = 0.0, work_pair = 0.0;
  for (int32_t i : order) {
    const double w = (double)ctxs[i]->Npad * ctxs[i]->Rpad * ctxs[i]->Ppad;
    work += w;
    if (ctxs[i]->tune.maximize_pair) work_pair += w;
  }
  b->pair = work_pair * 2.0 >= work;
  for (int32_t i : order) {
    const emc_context* c = ctxs[i];
    if (b->pair)
      banded((c->Npad + 255) / 256, c->Rpad / 256, c->tune.maximize_raster,
             [&](int64_t m, int64_t nt) {
               mt.push_back(TileDesc{(int32_t)(m * 256), 0, (int32_t)(nt * 256), 0,
                                     (int32_t)(c->Ppad / kPairBoxK), (int32_t)nt, (int32_t)m, i});
             });
    else
      banded(c->Npad / 128, c->Rpad / 256, c->tune.maximize_raster, [&](int64_t m, int64_t nt) {
        mt.push_back(TileDesc{(int32_t)(m * 128), 0, (int32_t)(nt * 256), 0,
                              (int32_t)(c->Ppad / kMaximizeBK), (int32_t)nt, (int32_t)m, i});
      });
  }
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t x, int32_t y) { return ctxs[x]->Npad > ctxs[y]->Npad; });
  double cwork_pair = 0.0;
  for (int32_t i : order)
    if (ctxs[i]->tune.compress_pair)
      cwork_pair += (double)ctxs[i]->Npad * ctxs[i]->Rpad * ctxs[i]->Ppad;
  b->cmp_pair = cwork_pair * 2.0 >= work;
  for (int32_t i : order) {
    const emc_context* c = ctxs[i];
    if (b->lists[i]) continue;
    if (b->cmp_pair)
      banded(c->Ppad / 256, c->Rpad / 256, c->tune.compress_raster, [&](int64_t nt, int64_t m) {
        ct.push_back(TileDesc{(int32_t)(m * 256), 0, (int32_t)(nt * 256), 0,
                              (int32_t)(c->Npad / kPairBoxK), (int32_t)nt, (int32_t)m, i});
      });
    else
      banded(c->Ppad / 256, c->Rpad / 128, c->tune.compress_raster, [&](int64_t nt, int64_t m) {
        ct.push_back(TileDesc{(int32_t)(m * 128), 0, (int32_t)(nt * 256), 0,
                              (int32_t)(c->Npad / kCompressBK), (int32_t)nt, (int32_t)m, i});
      });
  }
  b->n_mt = (int64_t)mt.size();
  b->n_ct = (int64_t)ct.size();
  mt.resize(std::max<size_t>(mt.size(), 1));  // no merged dataset: a list never read
  ct.resize(std::max<size_t>(ct.size(), 1));
  std::vector<MaxEpiArgs> me(n);
  std::vector<CmpEpiArgs> ce(n);
  for (int32_t i = 0; i < n; ++i) {
    me[i] = max_args(ctxs[i]);
    ce[i] = cmp_args(ctxs[i]);
  }
  emc_status s = EMC_OK;
  if ((s = b->cuda(cudaMalloc(&b->d_max, sizeof(MaxEpiArgs) * n), "cudaMalloc")) != EMC_OK ||
      (s = b->cuda(cudaMalloc(&b->d_cmp, sizeof(CmpEpiArgs) * n), "cudaMalloc")) != EMC_OK ||
      (s = b->cuda(cudaMemcpy(b->d_max, me.data(), sizeof(MaxEpiArgs) * n,
                              cudaMemcpyHostToDevice), "epilogue arguments")) != EMC_OK ||
      (s = b->cuda(cudaMemcpy(b->d_cmp, ce.data(), sizeof(CmpEpiArgs) * n,
                              cudaMemcpyHostToDevice), "epilogue arguments")) != EMC_OK ||
      (s = b->cuda(cudaMalloc(&b->d_mt, sizeof(TileDesc) * mt.size()), "cudaMalloc")) != EMC_OK ||
      (s = b->cuda(cudaMalloc(&b->d_ct, sizeof(TileDesc) * ct.size()), "cudaMalloc")) != EMC_OK ||
      (s = b->cuda(cudaMemcpy(b->d_mt, mt.data(), sizeof(TileDesc) * mt.size(),
                              cudaMemcpyHostToDevice), "tile list")) != EMC_OK ||
      (s = b->cuda(cudaMemcpy(b->d_ct, ct.data(), sizeof(TileDesc) * ct.size(),
                              cudaMemcpyHostToDevice), "tile list")) != EMC_OK) {
    emc_batch_destroy(b);
    return s;
  }
  *out = b;
  return EMC_OK;
}

emc_status emc_batch_iterate(emc_batch* b) {
  StageRange range("emc batch iteration");
  if (!b) return EMC_ERR_ARG;
  const int n = (int)b->ctx.size();
  emc_context* c0 = b->ctx[0];
  for (int i = 0; i < n; ++i)
    if (b->ctx[i]->stage != 0) return b->fail(EMC_ERR_STATE, "a dataset is between stages");
  // datasets with their own launches: one whole iteration each, in the order
  // a dataset iterated alone runs its stages
  for (int i = 0; i < n; ++i) {
    if (!b->alone[i]) continue;
    emc_context* c = b->ctx[i];
    BTRY(b, c, emc_expand(c));
    BCK(b, cudaMemcpyAsync(c->d_scaling_prev, c->d_scaling, sizeof(float) * c->N,
                           cudaMemcpyDeviceToDevice, b->st));
    emc_status s = batch_own_maximize(b, i);
    if (s == EMC_OK) s = batch_resp(b, i);
    if (s == EMC_OK) s = batch_own_compress(b, i);
    if (s != EMC_OK) return s;
    c->stage = 3;
    BTRY(b, c, emc_normalize(c));
  }
  if (b->n_mt == 0) return EMC_OK;  // no dataset shares the batched launches
  // the others through the batched launches (unused sets of the tensor-map
  // parameter repeat the first shared dataset's; no tile indexes them)
  int first = 0;
  while (b->alone[first]) ++first;
  TmapSet<kMaxBatch> maps;
  BatchMaxArgs me{};
  BatchCmpArgs ce{};
  me.tiles = b->d_mt;
  me.set = b->d_max;
  ce.tiles = b->d_ct;
  ce.set = b->d_cmp;
  for (int i = 0; i < n; ++i) {
    if (b->alone[i]) continue;
    emc_context* c = b->ctx[i];
    BTRY(b, c, emc_expand(c));
    BCK(b, cudaMemcpyAsync(c->d_scaling_prev, c->d_scaling, sizeof(float) * c->N,
                           cudaMemcpyDeviceToDevice, b->st));
  }
  for (int i = 0; i < kMaxBatch; ++i) {
    const emc_context* c = b->ctx[i < n && !b->alone[i] ? i : first];
    maps.a0[i] = b->pair ? c->tmKh64 : c->tmKh;
    maps.a1[i] = maps.a0[i];
    maps.b0[i] = b->pair ? c->tmBhi64 : c->tmBhi;
    maps.b1[i] = b->pair ? c->tmBlo64 : c->tmBlo;
  }
  if (b->pair)
    BCK(b, launch_batch_maximize_pair_tc(maps, b->n_mt, me, c0->d_status, c0->num_sms, b->st));
  else
    BCK(b, launch_batch_maximize_tc(maps, b->n_mt, me, c0->d_status, c0->num_sms, b->st));
  c0->launches += 1;
  for (int i = 0; i < n; ++i) {
    if (b->alone[i]) continue;
    const emc_status s = batch_resp(b, i);
    if (s != EMC_OK) return s;
  }
  if (b->n_ct) {
    for (int i = 0; i < kMaxBatch; ++i) {
      const emc_context* c = b->ctx[i < n && !b->alone[i] ? i : first];
      maps.a0[i] = c->tmPhi;
      maps.a1[i] = c->tmPlo;
      maps.b0[i] = b->cmp_pair ? c->tmKt128 : c->tmKt;
      maps.b1[i] = maps.b0[i];
    }
    if (b->cmp_pair)
      BCK(b, launch_batch_compress_pair_tc(maps, b->n_ct, ce, c0->d_status, c0->num_sms, b->st));
    else
      BCK(b, launch_batch_compress_tc(maps, b->n_ct, ce, c0->d_status, c0->num_sms, b->st));
    c0->launches += 1;
  }
  for (int i = 0; i < n; ++i) {
    if (b->alone[i] || !b->lists[i]) continue;
    const emc_status s = batch_own_compress(b, i);
    if (s != EMC_OK) return s;
  }
  for (int i = 0; i < n; ++i) {
    if (b->alone[i]) continue;
    emc_context* c = b->ctx[i];
    c->stage = 3;
    BTRY(b, c, emc_normalize(c));
  }
  return EMC_OK;
}

emc_status emc_batch_capture(emc_batch* b) {
  if (!b) return EMC_ERR_ARG;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  std::vector<int64_t> l0;
  std::vector<bool> prof;
  for (emc_context* c : b->ctx) {
    l0.push_back(c->launches);
    prof.push_back(c->prof);
    c->prof = false;  // no stage events inside the graph
  }
  BCK(b, cudaStreamSynchronize(b->st));
  BCK(b, cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
  const emc_status s = emc_batch_iterate(b);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->st, &g);
  b->per_iter.assign(b->ctx.size(), 0);
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    b->ctx[i]->prof = prof[i];
    b->per_iter[i] = b->ctx[i]->launches - l0[i];  // counted per replay instead
    b->ctx[i]->launches = l0[i];                    // captured, not launched
  }
  if (s != EMC_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  BCK(b, e);
  b->graph = g;
  BCK(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
  // the per-launch bookkeeping of one iteration, applied per replay
  for (emc_context* c : b->ctx) c->stage = 0;
  return EMC_OK;
}

emc_status emc_batch_launch(emc_batch* b, int32_t iterations) {
  if (!b || iterations < 0) return EMC_ERR_ARG;
  if (!b->exec) return b->fail(EMC_ERR_STATE, "emc_batch_capture first");
  for (int32_t k = 0; k < iterations; ++k) BCK(b, cudaGraphLaunch(b->exec, b->st));
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    emc_context* c = b->ctx[i];
    c->launches += b->per_iter[i] * iterations;
    c->resp_source = 1;
    c->stage = 0;
  }
  return EMC_OK;
}

emc_status emc_batch_synchronize(emc_batch* b) {
  if (!b) return EMC_ERR_ARG;
  BCK(b, cudaStreamSynchronize(b->st));
  for (emc_context* c : b->ctx) BTRY(b, c, check_status(c));
  // a dataset whose compacted entries passed the capacity ran the dense
  // compress (correct, slower): room for them from the next iteration on,
  // and a recorded graph is recorded again with the new buffers
  bool grew = false;
  for (size_t i = 0; i < b->ctx.size(); ++i) {
    emc_context* c = b->ctx[i];
    if (!b->lists[i]) continue;
    unsigned long long n = 0;
    BCK(b, cudaMemcpy(&n, c->d_lcount, sizeof(n), cudaMemcpyDeviceToHost));
    if ((int64_t)n > c->lcomp_cap) {
      BTRY(b, c, batch_lists_ready(c, (int64_t)n));
      grew = true;
    }
  }
  if (grew && b->exec) return emc_batch_capture(b);
  return EMC_OK;
}

void* emc_batch_stream(emc_batch* b) { return b ? (void*)b->st : nullptr; }

const char* emc_batch_last_error(const emc_batch* b) { return b ? b->err.c_str() : ""; }

}  // extern "C"
