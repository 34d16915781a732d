/*
 * emc_b200.h -- context API of the B200 EMC engine (libemc_b200.so).
 *
 * One context holds one dataset resident in HBM: detector geometry and mask,
 * rotation table, photon-count patterns, model, weight grid and per-pattern
 * scaling.  emc_iterate() runs one expand -> maximize -> compress iteration
 * in the order of the reference's main loop (emc.c:989-1084) on the
 * context's CUDA stream.
 *
 * Compared to the reference's API (include/emc.h) it adds: status codes on
 * every call, 64-bit sizes, a poisson likelihood and trilinear interpolation
 * next to the reference's gaussian / nearest-voxel ones, and a mixed-precision
 * tensor-core path (tcgen05, FP16 hi+lo operands, FP32 accumulation, FP64
 * log-sum-exp and normalisation).  All pointers are host pointers unless a
 * function says otherwise.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  EMC_OK = 0,
  EMC_ERR_ARG = 1,      /* invalid argument or size */
  EMC_ERR_CUDA = 2,     /* CUDA runtime error (emc_last_error has the text) */
  EMC_ERR_OOM = 3,      /* device allocation failed */
  EMC_ERR_TIMEOUT = 4,  /* a bounded device-side wait gave up (kernel returned early) */
  EMC_ERR_STATE = 5,    /* call out of order (e.g. iterate before set_patterns) */
  EMC_ERR_RANGE = 6,    /* data outside what the selected precision represents exactly */
  EMC_ERR_UNSUPPORTED = 7
} emc_status;

enum { EMC_LL_GAUSS = 0, EMC_LL_POISSON = 1 };
enum { EMC_INTERP_NEAREST = 0, EMC_INTERP_TRILINEAR = 1 };
enum { EMC_PREC_FP32 = 0, EMC_PREC_MIXED = 1 };

typedef struct {
  int32_t side;         /* detector side in pixels == model side in voxels */
  int32_t likelihood;   /* EMC_LL_* */
  int32_t interp;       /* EMC_INTERP_* */
  int32_t precision;    /* EMC_PREC_* */
  int64_t n_patterns;
  int64_t n_rotations;
  float sigma;          /* gaussian width (reference emc.c:734 uses 0.4) */
  float poisson_floor;  /* lower bound of W inside log W (poisson) */
  int32_t device;       /* CUDA device ordinal */
  int32_t flags;        /* reserved, 0 */
} emc_config;

typedef struct {
  double sum_plogp;     /* sum P log P: the value emc.c:1018 logs as "likelihood" */
  double total_loglik;  /* sum_p logsumexp_r LL_rp, FP64 */
  double model_max;     /* after normalisation */
  double total_resp;    /* sum_r T_r (== number of patterns) */
} emc_iter_stats;

typedef struct emc_context emc_context;

/* Buffers readable with emc_get_buffer (host copy) / emc_device_buffer. */
typedef enum {
  EMC_BUF_MODEL = 0,    /* float [side^3] */
  EMC_BUF_WEIGHT = 1,   /* float [side^3] weight grid of the last compress */
  EMC_BUF_SCALING = 2,  /* float [N] */
  EMC_BUF_RESP = 3,     /* float [R][N] responsibilities after maximize (after a proposed
                           iteration: 0 outside each pattern's candidate cells; host copy only) */
  EMC_BUF_SLICES = 4,   /* float [R][Pa] expanded slices (FP32 path), Pa = active pixels */
  EMC_BUF_TOTALRESP = 5, /* float [R] T_r */
  EMC_BUF_ACCUM = 6,     /* float [2*side^3] insertion accumulators (model and weight sums)
                            between emc_compress_insert and emc_normalize */
  EMC_BUF_TOTALRESP_ALL = 7 /* float [R] T_r for the insertion's T_r <= 1e-10 skip: after
                            maximize a copy of this context's T_r; a caller sharding the
                            patterns over contexts replaces it by the sum over all of them */
} emc_buffer;

const char *emc_status_string(emc_status s);
/* Text of the last error on this context (or of the last failed emc_create). */
const char *emc_last_error(const emc_context *ctx);

emc_status emc_create(const emc_config *cfg, emc_context **out);
emc_status emc_destroy(emc_context *ctx);

/* Pixel coordinates (emc.c:365-393 layout, [y*side+x]) and mask.  Pixels with
 * mask != 0 enter the likelihood and scaling; mask == 1 pixels are inserted
 * (emc_cuda.cu:120, emc_atomic.cu:30). */
emc_status emc_set_geometry(emc_context *ctx, const float *x, const float *y, const float *z,
                            const int32_t *mask);
/* Unit quaternions [R][4] and rotation weights [R]. */
emc_status emc_set_rotations(emc_context *ctx, const float *quaternions, const float *weights);
/* Photon counts [N][side*side]: finite and non-negative (EMC_ERR_RANGE
 * otherwise); the mixed path needs integers <= 2048.  A rejected upload
 * leaves the context without patterns.  emc_set_model rejects NaN or
 * infinite values, emc_set_scaling anything but finite positive numbers,
 * emc_set_rotations non-finite quaternions or negative weights, and
 * emc_set_geometry non-finite coordinates (all EMC_ERR_RANGE). */
emc_status emc_set_patterns(emc_context *ctx, const float *counts);
/* The same from photon lists (sparse patterns, CSR over patterns): pattern p's
 * entries are row_ptr[p] .. row_ptr[p+1]-1 (row_ptr[0] = 0, row_ptr[N] =
 * entry count); pixels[e] is a detector pixel index (y * side + x) and
 * counts[e] its count, or counts = NULL for one photon per entry (a pixel
 * may repeat).  Entries on masked-out pixels are dropped; entries outside
 * the detector are an error.  Only the lists cross the bus. */
emc_status emc_set_patterns_sparse(emc_context *ctx, const int64_t *row_ptr,
                                   const int32_t *pixels, const float *counts);
emc_status emc_set_model(emc_context *ctx, const float *model);
emc_status emc_set_scaling(emc_context *ctx, const float *scaling);

/* One iteration.  stats may be NULL; with stats the call waits for the
 * iteration, without it the work is only enqueued on the context stream. */
emc_status emc_iterate(emc_context *ctx, emc_iter_stats *stats);
/* Stage-by-stage form of emc_iterate (the three calls in order == one iteration). */
emc_status emc_expand(emc_context *ctx);
emc_status emc_maximize(emc_context *ctx);
emc_status emc_compress(emc_context *ctx);
/* emc_compress in two halves: insertion into the accumulators
 * (EMC_BUF_ACCUM), then model = sum / weight normalised to mean 1.  Between
 * them a pattern-sharded run sums the accumulators across ranks (the only
 * exchange of an EMC iteration: every other quantity is per pattern or per
 * rotation). */
emc_status emc_compress_insert(emc_context *ctx);
emc_status emc_normalize(emc_context *ctx);
/* sum P log P and sum_p lse_p of this context's patterns in the last iteration. */
emc_status emc_partial_stats(emc_context *ctx, double *sum_plogp, double *total_loglik);

emc_status emc_synchronize(emc_context *ctx);
emc_status emc_get_model(emc_context *ctx, float *model);
emc_status emc_get_scaling(emc_context *ctx, float *scaling);
emc_status emc_get_buffer(emc_context *ctx, emc_buffer which, void *host, size_t bytes);
/* The responsibilities of n chosen patterns (indices patterns[n]) from the
 * last maximize, dense or proposed, into the host array out [R][n] (column a
 * is pattern patterns[a]; 0 outside a proposed iteration's candidates). */
emc_status emc_get_resp_columns(emc_context *ctx, int64_t n, const int64_t *patterns, float *out);
/* Device pointer of a buffer (valid until emc_destroy). */
emc_status emc_device_buffer(emc_context *ctx, emc_buffer which, void **dptr, size_t *bytes);
/* Per-stage device timing.  With profiling on, every iteration records CUDA
 * events around its stages.  emc_stage_times returns milliseconds of
 * [expand, maximize contraction, responsibility pass (softmax + scaling),
 * compress contraction + insertion, normalisation] of the previous profiled
 * iteration (of the only one after the first), waiting for it if needed, so
 * it can be called after each emc_iterate without draining the stream. */
emc_status emc_set_profiling(emc_context *ctx, int on);
emc_status emc_stage_times(emc_context *ctx, float ms[5]);
/* Cap on the device memory this context allocates, in bytes (0: no cap; the
 * default).  A call whose allocations would pass it fails with EMC_ERR_OOM
 * before allocating; the context is then only good for emc_destroy, which
 * frees what it holds.  EMC_ERR_ARG when the cap is below what is already
 * held.  emc_memory_used: device bytes the context holds. */
emc_status emc_set_memory_limit(emc_context *ctx, size_t bytes);
size_t emc_memory_used(const emc_context *ctx);
/* Rotation chunks (mixed contexts).  The log-likelihood Y of a dense
 * iteration takes R x N x 4 bytes; with chunks of `rows` rotations (a
 * multiple of 256) Y holds one chunk at a time: per chunk the contraction,
 * an online log-sum-exp over the tile partials of the chunks so far, and a
 * sweep that keeps every entry whose responsibility under that running
 * log-sum-exp is at least 1e-30 (it can only fall later).  The last chunk's
 * log-sum-exp is final; lse, scaling and sum P log P are those of the
 * unchunked iteration, and the compress reads the responsibility lists
 * formed from the kept entries (the dense compress operand P' is not
 * allocated).  The last chunk holds the remainder (uneven).
 * rows: 0 = one chunk of every rotation; -1 = the most rotations whose Y
 * fits in half of what the memory limit and the free device memory leave.
 * capacity: entries the kept-entry arrays start with (0: max(64 N, 2^20));
 * an iteration that keeps more grows them and runs its chunks again.  In a
 * batch (rows 0) it is the first capacity of the responsibility lists.
 * emc_set_geometry already chooses chunks (rows -1) when Y and P' of every
 * rotation do not fit.  EMC_ERR_UNSUPPORTED for FP32 contexts and above
 * 51,200 active pixels (the responsibility lists' limit); EMC_ERR_STATE
 * inside an iteration or a batch (a batch takes unchunked contexts only).
 * After a chunked iteration the responsibilities are read as usual
 * (emc_get_buffer EMC_BUF_RESP, emc_get_resp_columns, emc_orientation_stats,
 * emc_cell_targets, emc_cell_log_mass) from the kept entries, 0 elsewhere.
 * emc_rotation_chunk: the rotations Y holds (R when unchunked). */
emc_status emc_set_rotation_chunk(emc_context *ctx, int64_t rows, int64_t capacity);
int64_t emc_rotation_chunk(const emc_context *ctx);
/* Deterministic insertion (on = 1): every insertion sum (model and weight per
 * voxel) is formed exactly as a fixed-point integer (64 fraction bits, 32-bit
 * pieces added to 64-bit limbs; integer addition does not depend on order)
 * and rounded once; the responsibility lists are sorted by (rotation,
 * pattern) and each rotation's slice sums its patterns in that order.  Two
 * runs of the same iterations then give bitwise the same model, weight and
 * scaling, chunked or not, in either precision.  Costs 64 bytes of device
 * memory per voxel.  EMC_ERR_UNSUPPORTED for the proposed iterations; a
 * batch takes contexts without it. */
emc_status emc_set_deterministic(emc_context *ctx, int on);
/* Checkpoint (emc.c:715-716 resumes from a model file at start_iteration;
 * this keeps the whole state): model, weight grid and per-pattern scaling
 * with the iteration number, in a raw little-endian file.  The model and the
 * scaling are everything the next iteration reads, so a context loaded from
 * the file continues exactly as the saved one would.  Loading needs the same
 * side, pattern and rotation counts (EMC_ERR_RANGE otherwise); the
 * likelihood, interpolation and precision may differ. */
emc_status emc_save_state(emc_context *ctx, const char *path, int64_t iteration);
emc_status emc_load_state(emc_context *ctx, const char *path, int64_t *iteration);
/* Number of kernels this context has launched since creation. */
int64_t emc_launch_count(const emc_context *ctx);
/* cudaStream_t the context enqueues on. */
void *emc_stream(emc_context *ctx);
/* Number of active (mask != 0) pixels. */
int64_t emc_active_pixels(const emc_context *ctx);

/* Orientation diagnostics of the last maximize (dense or proposed), host
 * outputs, each optional: best_rot[N] the most probable rotation of every
 * pattern (for a proposed iteration: among its candidates) and best_resp[N]
 * its responsibility; avg_resp[R] the average responsibility of each
 * rotation over the patterns (T_r / N).  The per-iteration record the
 * reference's viewer reads (best rotations, average_resp, scaling). */
emc_status emc_orientation_stats(emc_context *ctx, int32_t *best_rot, float *best_resp,
                                 float *avg_resp);

/* ---- several datasets in one launch ----
 * Up to 8 mixed-precision contexts on one device (each set up with its own
 * geometry, rotations, patterns and model; detector sizes may differ) iterate
 * together: both contractions run as one persistent launch over a tile list
 * spanning the datasets (costliest tiles first), the per-dataset stages
 * between them on one shared stream.  A dataset whose maximize alone fills
 * the GPU for eight waves of tiles keeps its own contraction launches in the
 * same stream and graph.  A dataset with responsibility lists
 * (emc_set_tuning compress_sparse) compresses from them with their count kept
 * on the device: past their capacity that iteration runs its dense compress
 * instead, and emc_batch_synchronize gives the lists room (recording a
 * captured graph again).  The contexts keep that stream until
 * emc_batch_destroy; their own calls (get_model, ...) stay ordered with the
 * batch.  emc_batch_capture records one batched iteration into a CUDA graph;
 * emc_batch_launch replays it.  Destroy a batch before its contexts. */
typedef struct emc_batch emc_batch;
emc_status emc_batch_create(emc_context *const *ctxs, int32_t n, emc_batch **out);
emc_status emc_batch_destroy(emc_batch *batch);
/* Enqueue one iteration of every dataset (no host synchronisation). */
emc_status emc_batch_iterate(emc_batch *batch);
emc_status emc_batch_capture(emc_batch *batch);
emc_status emc_batch_launch(emc_batch *batch, int32_t iterations);
/* Wait for the batch's stream; reports device wait timeouts of its kernels;
 * grows the lists of a dataset that overflowed them (see above). */
emc_status emc_batch_synchronize(emc_batch *batch);
void *emc_batch_stream(emc_batch *batch);
const char *emc_batch_last_error(const emc_batch *batch);

/* Tile order of the two tensor-core contractions (mixed precision): the
 * persistent CTAs walk the output tiles in bands of `raster` rotation tiles,
 * the other index fastest, so operand tiles loaded from HBM are shared
 * through L2 by the CTAs in flight.  1 = plain row order. */
typedef struct {
  int32_t maximize_raster, compress_raster;
  int32_t maximize_pair; /* 1: the maximize contraction on SM pairs (cta_group::2) */
  int32_t compress_pair; /* 1: the compress contraction on SM pairs */
  int32_t maximize_sparse; /* FP32 poisson contexts: 1 = the log-likelihood as a
                              photon-list gather over each pattern's non-zero pixels
                              instead of the dense contraction */
  int32_t compress_sparse; /* FP32 contexts: 1 = the slice sums as a gather over each
                              pixel's non-zero counts instead of the dense contraction */
} emc_tuning;
/* Time-out check (no counterpart in the reference): runs one bounded device
 * wait on an mbarrier that nothing completes, given up after limit_us
 * microseconds (1 .. 1,000,000), through the same wait routine as every
 * tensor-core kernel.  Returns EMC_ERR_TIMEOUT with the wait site (90) in
 * emc_last_error; the status word is cleared and the context stays usable. */
emc_status emc_wait_probe(emc_context *ctx, uint32_t limit_us);
emc_status emc_get_tuning(const emc_context *ctx, emc_tuning *t);
emc_status emc_set_tuning(emc_context *ctx, const emc_tuning *t);
/* Autotuner: two iterations per candidate band size (the maximize on one SM
 * and on SM pairs; both contractions timed by stage events) from the current
 * model and scaling, which are restored afterwards; keeps the fastest band
 * size of each contraction and the faster maximize form.  ms (optional):
 * [2][n], the best maximize then compress time per candidate.  FP32
 * contexts: one iteration with the dense contractions and one with the
 * photon-list forms (maximize_sparse for poisson, compress_sparse), keeping
 * the faster form of each; the candidates are not used and ms[0] / ms[n]
 * receive the chosen maximize / compress times. */
emc_status emc_autotune(emc_context *ctx, const int32_t *candidates, int32_t n, float *ms,
                        emc_tuning *best);

/* ---- learned rotation proposal ----
 * Fine rotations are grouped into coarse cells (e.g. the nearest rotation of
 * the 420-rotation 600-cell sampling); the rotation list given to
 * emc_set_rotations must be sorted by cell.  A proposal network predicts, per
 * pattern, a posterior over the cells; emc_iterate_proposed then evaluates
 * each pattern only against the fine rotations of its most probable cells,
 * or runs the dense iteration when the mean predicted mass on those cells is
 * below `threshold`. */
typedef struct {
  double mean_mass, min_mass;  /* predicted posterior mass on the evaluated cells */
  int64_t pairs;               /* (pattern, cell) pairs evaluated */
  int64_t evaluations;         /* (pattern, rotation) evaluations */
  int32_t fallback;            /* 1: the dense iteration ran instead */
  int32_t audited;             /* patterns evaluated against every rotation (emc_iterate_topk) */
  double sum_plogp, total_loglik;
  /* share of each audited pattern's responsibility (against every rotation)
   * that its candidate cells hold: mean and minimum over the audited patterns */
  double audit_mean_captured, audit_min_captured;
} emc_proposal_stats;

/* cell[r] for every rotation (non-decreasing), n_cells cells. */
emc_status emc_set_cells(emc_context *ctx, const int32_t *cell, int32_t n_cells);
/* x [N][in_side^2] (device): log(1 + counts summed over 2x2 pixel blocks),
 * in_side = side / 2; the proposal network's input. */
emc_status emc_pattern_features(emc_context *ctx, int32_t in_side, float *x_device);
/* t [N][n_cells] (device): the responsibilities of the last maximize (dense,
 * or proposed: then 0 outside each pattern's candidate cells) summed over
 * each cell's rotations; the proposal network's training target. */
emc_status emc_cell_targets(emc_context *ctx, float *t_device);
/* One iteration restricted, per pattern, to candidate cells: with
 * keep_device (optional, [N][n_cells], e.g. the previous iteration's
 * emc_cell_targets) first the most probable cells under keep that hold
 * keep > 0, until at least min_cells are taken and their keep mass reaches
 * keep_mass; then cells in order of cell_probs (the proposal) until at least
 * min_cells are taken and their cell_probs mass reaches mass_target (>= 1:
 * always max_cells cells), at most max_cells in all
 * (1 <= min_cells <= max_cells).  The dense iteration runs instead when the
 * mean cell_probs mass of the candidates is below `threshold`.
 * cell_probs: device [N][n_cells]. */
emc_status emc_iterate_proposed(emc_context *ctx, const float *cell_probs_device,
                                const float *keep_device, int32_t min_cells, int32_t max_cells,
                                float mass_target, float keep_mass, float threshold,
                                emc_proposal_stats *stats);

/* The proposal of the configuration "top-k fine rotations evaluated from the
 * coarse posterior, dense maximize when the captured responsibility falls
 * below a bound":
 *   - log_keep (optional, device [N][n_cells]): the log-posterior mass of
 *     every cell in a previous iteration (emc_cell_log_mass); each pattern
 *     takes its cells in that order (finite values only) until they hold at
 *     least top_k fine rotations and, with keep_tail > 0, all but keep_tail
 *     of that posterior;
 *   - cell_probs (optional, device [N][n_cells]): the proposal network's cell
 *     posterior; cells are then added in its order until the candidates'
 *     predicted mass reaches mass_target (every pattern gets at least one);
 *   - at most max_cells cells per pattern;
 *   - audit_patterns (0..128) patterns, an evenly strided sample shifted on
 *     every call, are evaluated against every rotation after the expansion;
 *     when one of them holds less than min_captured of its responsibility on
 *     its candidate cells, the dense iteration runs instead (stats->fallback,
 *     stats->audit_*).
 * At least one of log_keep and cell_probs is given. */
typedef struct {
  int32_t top_k;
  int32_t max_cells;
  float mass_target;
  int32_t audit_patterns;
  float min_captured;
  float keep_tail;  /* > 0: also keep taking log_keep cells until they hold all but this much
                       of the previous posterior (e.g. 1e-6); 0: top_k alone */
} emc_topk_config;
emc_status emc_iterate_topk(emc_context *ctx, const float *cell_probs_device,
                            const float *log_keep_device, const emc_topk_config *cfg,
                            emc_proposal_stats *stats);
/* t [N][n_cells] (device): natural log of each cell's responsibility mass in
 * the last maximize (dense, or proposed: -inf outside the candidate cells),
 * formed in the log domain (the cell's largest log-likelihood plus the log of
 * an FP64 sum relative to it), so every evaluated cell is ranked however far
 * down the tail it lies. */
emc_status emc_cell_log_mass(emc_context *ctx, float *t_device);

/* Proposal network: three 3x3 stride-2 convolutions (16, 32, 64 channels,
 * ReLU) and a fully connected layer to n_out logits, softmax.  BF16 weights
 * and activations (bf16 = 0: FP32, for gradient checks), FP32 accumulation,
 * FP32 master weights, Adam.  All data pointers are device pointers. */
typedef struct emc_net emc_net;
emc_status emc_net_create(int in_side, int n_out, int bf16, uint64_t seed, int device,
                          emc_net **out);
emc_status emc_net_destroy(emc_net *net);
int64_t emc_net_num_params(const emc_net *net);
emc_status emc_net_get_params(emc_net *net, float *host);
emc_status emc_net_set_params(emc_net *net, const float *host);
/* probs [batch][n_out] from x [batch][in_side^2]. */
emc_status emc_net_forward(emc_net *net, const float *x, int64_t batch, float *probs);
/* Mean soft-target cross-entropy of (x, t [batch][n_out]) and its gradient
 * (kept inside; copied to grad_host when not NULL, layout as the parameters). */
emc_status emc_net_gradients(emc_net *net, const float *x, const float *t, int64_t batch,
                             double *loss, float *grad_host);
/* emc_net_gradients followed by one Adam step with learning rate lr. */
emc_status emc_net_train_step(emc_net *net, const float *x, const float *t, int64_t batch,
                              float lr, double *loss);
const char *emc_net_last_error(const emc_net *net);

/* ---- host-side input generators (reference host code, C++ here) ---- */

int64_t emc_n_to_samples(int n); /* emc.c:43 */
/* 600-cell rotation sampling of emc.c:49-363.  halve != 0 keeps one quaternion
 * of each +-q pair (both give the same slice) and renormalises the weights.
 * Returns R, or -1 on failure; quaternions/weights may be NULL to query R. */
int64_t emc_generate_rotations(int n, int halve, float *quaternions, float *weights);
/* emc.c:365-393, arrays [y*side+x]. */
void emc_detector_coordinates(int side, double wavelength, double pixel_size,
                              double detector_distance, float *x, float *y, float *z);

typedef struct {
  int32_t side;
  int32_t n_scatterers;      /* point scatterers of unit strength */
  double object_radius;      /* sphere radius as a fraction of the box side */
  int64_t n_patterns;
  double mean_photons;       /* mean photons per pattern */
  double scale_sigma;        /* lognormal sigma of the per-pattern scale */
  double beamstop_radius;    /* pixels; mask = 0 within this radius */
  uint64_t seed;
  int64_t first_pattern;     /* index of counts[0] in the seeded pattern sequence (shards) */
} emc_synth_config;

/* Synthetic dataset: |F|^2 of point scatterers on a side^3 grid (model, may be
 * NULL), counts [N][side^2] drawn as Poisson(slice at a uniform random
 * rotation x mean_photons/sum(slice) x lognormal scale), mask [side^2],
 * true_rotations [N][4] and true_scales [N] (either may be NULL).
 * Coordinates x,y,z come from emc_detector_coordinates. */
emc_status emc_synthesize(const emc_synth_config *sc, const float *x, const float *y,
                          const float *z, float *true_model, float *counts, int32_t *mask,
                          float *true_rotations, float *true_scales);
/* Uniform [0,1) initial model (emc.c:893-898 with a counter-based generator). */
void emc_random_model(int side, uint64_t seed, float *model);
/* Initial model from the data (emc.c:896-914, model_input 1): every image
 * inserted with weight 1 at a uniformly random rotation (nearest voxel,
 * mask == 1), then model = sum / weight (0 where no weight).  images:
 * [n_images][side^2]; quat_out (optional): the rotations used, [n][4]. */
emc_status emc_model_random_orientations(int side, int64_t n_images, const float *images,
                                         const int32_t *mask, const float *x, const float *y,
                                         const float *z, uint64_t seed, float *model,
                                         float *quat_out);
/* Model from / to a file (emc.c:915-925, model_input 2): raw little-endian
 * float32, side^3 values in [z][y][x] order; load keeps |value|.
 * EMC_ERR_RANGE when the file size is not 4 side^3 bytes. */
emc_status emc_model_load(const char *path, int side, float *model);
emc_status emc_model_save(const char *path, int side, const float *model);

#ifdef __cplusplus
}
#endif
