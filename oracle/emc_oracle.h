/*
 * EMC FP64 oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A CPU restatement (C++17 + OpenMP, FP64 arithmetic) of the reference's
 * expand -> maximize -> compress iteration.  Only tests/, the smoke check and
 * bench.py's CPU-baseline / reference leg may load it; the product library
 * (emc_b200/) never links or calls it.
 *
 * Parity anchors (reference file:line, paths inside FilipeMaia/emc):
 *   rotations     emc.c:43-363      (600-cell sampling; halved to one of each +-q pair)
 *   coordinates   emc.c:365-393
 *   expand        emc_cuda.cu:51-111 (nearest, exclusive lower bound >0)
 *   log-likelihood emc_cuda.cu:113-150, emc.c:667-682 (gaussian "absolute")
 *   softmax       emc_cuda.cu:445-476
 *   scaling       emc_cuda.cu:195-228
 *   slice average emc_atomic.cu:76-113
 *   insertion     emc_atomic.cu:17-73,115-133 (nearest, inclusive lower bound >=0)
 *   normalise     emc_cuda.cu:414-433
 *   iteration     emc.c:989-1084
 * The poisson likelihood and trilinear interpolation are not in the reference;
 * they follow the equations stated beside each function below.
 *
 * Voxel choice is a discrete decision, so it is computed in FP32 with a fixed
 * operation order (no contraction except the explicit fmaf calls) exactly as
 * the CUDA kernels do; every other quantity is FP64.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_LL_GAUSS = 0, ORC_LL_POISSON = 1 };
enum { ORC_NEAREST = 0, ORC_TRILINEAR = 1 };

typedef struct {
  int32_t side;        /* detector side == model side */
  int32_t likelihood;  /* ORC_LL_* */
  int32_t interp;      /* ORC_NEAREST / ORC_TRILINEAR */
  int32_t pad_;
  int64_t n_patterns;
  int64_t n_rotations;
  double sigma;          /* gaussian width (emc.c:734) */
  double poisson_floor;  /* W floor inside log for the poisson likelihood */
} orc_config;

typedef struct {
  double sum_plogp;     /* sum P log P (what emc.c:1018 logs as "likelihood") */
  double total_loglik;  /* sum_p logsumexp_r LL_rp */
  double model_max;
  double total_resp;    /* sum_r T_r */
} orc_stats;

int64_t orc_n_to_samples(int n);
/* Generates the 600-cell sampling of emc.c:49-363.  q: [R][4], w: [R].
 * halve != 0 keeps one quaternion of each +-q pair and renormalises w.
 * Returns R; q/w may be NULL to query the count. */
int64_t orc_generate_rotations(int n, int halve, double* q, double* w);
/* emc.c:365-393; outputs indexed [y*side + x]. */
void orc_coordinates(int side, double wavelength, double pixel_size, double detector_distance,
                     double* x, double* y, double* z);
/* FP32 rotation matrix with the coefficient order of emc_cuda.cu:65-85. */
void orc_rotation_matrix_f32(const float* q, float* m);

/* S[r][i] for every pixel i (mask ignored, as in emc_cuda.cu:51-98). */
void orc_expand(const orc_config* c, const double* model, const float* rot,
                const float* cx, const float* cy, const float* cz, double* slices);
/* LL[r][p]. */
void orc_loglik(const orc_config* c, const double* slices, const float* images,
                const int32_t* mask, const double* scaling, double* ll);
/* Same, gaussian mode evaluated as the direct sum of squared differences. */
void orc_loglik_gauss_direct(const orc_config* c, const double* slices, const float* images,
                             const int32_t* mask, const double* scaling, double* ll);
/* In-place per-pattern softmax over r of resp[r][p]; lse[p] optional.
 * Returns sum P log P. */
double orc_softmax(int64_t R, int64_t N, double* resp, double* lse);
/* New per-pattern scaling (in place). */
void orc_update_scaling(const orc_config* c, const double* slices, const float* images,
                        const int32_t* mask, const double* resp, double* scaling);
/* U[r][i] = sum_p P_rp K_pi / phi_p (mask != 0, else 0); total_resp[r] = T_r. */
void orc_slice_average(const orc_config* c, const double* resp, const float* images,
                       const int32_t* mask, const double* scaling, double* U,
                       double* total_resp);
/* Inserts U/T with weight rotw*T into the accumulators (mask == 1 pixels). */
void orc_insert(const orc_config* c, const double* U, const double* total_resp,
                const int32_t* mask, const float* rot, const float* rotw, const float* cx,
                const float* cy, const float* cz, double* model_acc, double* weight_acc);
/* The same for one shard of the patterns: the T_r <= 1e-10 skip reads
   all_total_resp (T_r summed over every shard). */
void orc_insert_shard(const orc_config* c, const double* U, const double* total_resp,
                      const double* all_total_resp, const int32_t* mask, const float* rot,
                      const float* rotw, const float* cx, const float* cy, const float* cz,
                      double* model_acc, double* weight_acc);
/* Slice average + insertion into zeroed accumulators; total_resp[r] = T_r. */
void orc_compress(const orc_config* c, const double* resp, const float* images,
                  const int32_t* mask, const double* scaling, const float* rot,
                  const float* rotw, const float* cx, const float* cy, const float* cz,
                  double* model_acc, double* weight_acc, double* total_resp);
/* model = model/weight (0 where weight==0), then model /= mean(model). */
void orc_normalize_model(int64_t M, double* model, const double* weight);
/* One full iteration in the order of emc.c:989-1084. resp_out: optional [R][N]. */
void orc_iterate(const orc_config* c, const float* images, const int32_t* mask,
                 const float* rot, const float* rotw, const float* cx, const float* cy,
                 const float* cz, double* model, double* scaling, double* resp_out,
                 orc_stats* stats);
/* The same iteration with the softmax restricted, per pattern, to a candidate
   set of rotations: allowed[r][p] != 0 (every pattern needs at least one).
   Log-likelihoods outside the set are -inf, so those responsibilities are 0
   and the scaling update and compress sum over the candidates only.  This is
   the iteration the learned orientation proposal evaluates (a top-k of the
   rotations per pattern); with every pair allowed it equals orc_iterate. */
void orc_iterate_restricted(const orc_config* c, const float* images, const int32_t* mask,
                            const float* rot, const float* rotw, const float* cx, const float* cy,
                            const float* cz, const uint8_t* allowed, double* model,
                            double* scaling, double* resp_out, orc_stats* stats);

/* Seeded synthetic inputs (the benchmark configurations' data): a uniform
 * [0,1) model, and a dataset of point-scatterer |F|^2 (true_model, optional),
 * beamstop mask [side^2] and Poisson counts [n_patterns][side^2] drawn at
 * uniform random rotations with lognormal scales; patterns first_pattern ..
 * first_pattern + n_patterns - 1 of the seeded sequence.  Returns 0, or 1 for
 * invalid arguments. */
void orc_random_model(int side, uint64_t seed, float* model);
int orc_synthesize(int side, int n_scatterers, double object_radius, int64_t n_patterns,
                   double mean_photons, double scale_sigma, double beamstop_radius,
                   uint64_t seed, int64_t first_pattern, const float* x, const float* y,
                   const float* z, float* true_model, float* counts, int32_t* mask);

#ifdef __cplusplus
}
#endif
