/*
 * emc.h -- drop-in replacement for FilipeMaia/emc's C host API (emc.h:1-59).
 *
 * Same names, argument order and meaning as the reference; link
 * libemc_b200.so instead of emc_cuda.o + emc_atomic.o.  Every function keeps
 * the reference's synchronous behaviour (it returns after its device work and
 * any host copy it documents are complete).  The engine behind them is the
 * FP32 CUDA-core path of libemc_b200 (gaussian "absolute" likelihood,
 * nearest-voxel slicing), written for sm_100a.
 *
 * Types: the reference takes real/sp_matrix/sp_3matrix/sp_imatrix from
 * libspimage.  Define EMC_HAVE_SPIMAGE before including this header to use
 * <spimage.h>; otherwise the layout-compatible subset below is used (only
 * `data` and the dimensions are ever read).
 */
#pragma once

#ifdef EMC_HAVE_SPIMAGE
#include <spimage.h>
#else
typedef float real;
typedef struct { unsigned int rows, cols; real *data; } sp_matrix;        /* (row,col) at data[col*rows+row] */
typedef struct { unsigned int rows, cols; int *data; } sp_imatrix;
typedef struct { unsigned int x, y, z; real *data; } sp_3matrix;          /* (x,y,z) at data[(z*y_dim+y)*x_dim+x] */
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* emc.h:8-10 */
typedef struct {
  real q[4];
} Quaternion;

/* emc.h:12-18 */
typedef struct {
  int side;
  real wavelength;
  real pixel_size;
  int detector_size;
  real detector_distance;
} Setup;

/* emc.h:20-22 (reference CPU routine, emc.c:491-539): nearest-voxel insertion of
 * one slice with weight w, mask == 1 pixels only, host memory. */
void insert_slice(sp_3matrix *model, sp_3matrix *weight, sp_matrix *slice, sp_imatrix *mask,
                  real w, Quaternion *rot, sp_matrix *x_coordinates, sp_matrix *y_coordinates,
                  sp_matrix *z_coordinates);

/* emc.h:24-29 (emc_cuda.cu:292-362): slice average of every rotation from the
 * responsibilities and the current scaling, insertion into d_model/d_weight
 * (which the caller zeroed with cuda_reset_model), copy of d_model into
 * model->data.  `weights` is the host array of rotation weights.  Returns
 * sum_r T_r.  d_slices is overwritten with the averaged slices. */
real cuda_update_slices(real *d_images, real *slices, int *d_mask, real *d_respons,
                        real *d_scaling, int N_images, int N_slices, int N_2d,
                        sp_3matrix *model, real *d_model, real *x_coordinates,
                        real *y_coordinates, real *z_coordinates, real *d_rotations,
                        real *weights, real *d_weight, Setup setup, sp_matrix **images);

/* emc.h:32-34 (emc_cuda.cu:195-264): d_scaling[p] = sum_mask K^2 /
 * sum_r P_rp sum_mask K S_r; also copied into the host array `scaling`. */
void cuda_update_scaling(real *d_images, real *slices, int *d_mask, real *d_respons,
                         real *d_scaling, int N_images, int N_slices, int N_2d, real *scaling);

/* emc.h:35-37 (emc_cuda.cu:113-193): d_respons[r*N_images+p] =
 * -sum_mask (S_r - K_p/phi_p)^2 / (2 count sigma^2); also copied into `respons`. */
void cuda_calculate_responsabilities(real *slices, real *images, int *d_mask, real sigma,
                                     real *d_scaling, real *d_respons, int N_2d, int N_images,
                                     int N_slices, real *respons);

/* emc.h:39-41 (emc_cuda.cu:51-111,267-290): nearest-voxel slices of d_model. */
void cuda_get_slices(sp_3matrix *model, real *d_model, real *d_slices, real *d_rot,
                     real *d_x_coordinates, real *d_y_coordinates, real *d_z_coordinates,
                     int N_slices);

/* emc.h:43-56 (emc_cuda.cu:364-443,478-505) */
void cuda_allocate_slices(real **slices, Setup setup, int N_slices);
real cuda_model_max(real *model, int model_size);
void cuda_allocate_model(real **d_model, sp_3matrix *model);
void cuda_allocate_mask(int **d_mask, sp_imatrix *mask);
void cuda_reset_model(sp_3matrix *model, real *d_model);
void cuda_normalize_model(sp_3matrix *model, real *d_model, real *d_weight);
void cuda_allocate_rotations(real **d_rotations, Quaternion **rotations, int N_slices);
void cuda_allocate_images(real **d_images, sp_matrix **images, int N_images);
void cuda_allocate_coords(real **d_x, real **d_y, real **d_z, sp_matrix *x, sp_matrix *y,
                          sp_matrix *z);
void cuda_allocate_real(real **x, int n); /* n is a byte count, as in emc_cuda.cu:435-437 */
void cuda_allocate_scaling(real **scaling, int N_images);
void cuda_normalize_responsabilities(real *d_respons, int N_slices, int N_images);
real cuda_total_respons(real *d_respons, real *respons, int n);

/* No counterpart in the reference.  cuda_normalize_responsabilities followed
 * by cuda_total_respons, for callers that cannot call cudaMalloc: code that
 * runs while a stream is being captured into a CUDA graph, processes held to a
 * fixed device-memory budget, or an allocator-owning host framework that
 * forbids allocations behind its back.  The kernels' scratch (one FP64
 * partial per 32 patterns) is a fixed 512 KB array in the library's device
 * image instead of memory the library allocates, so this function allocates
 * nothing; every GPU that loads the library holds that array until exit.
 * Limit: N_images <= 2,097,152; larger calls are rejected with status 1.
 * d_respons [N_slices][N_images] is normalised in place on `stream` (a
 * cudaStream_t, NULL for the default stream).  sum_plogp (optional)
 * receives sum P log P:
 *   - a device (or managed) pointer: written by a kernel on `stream`; the call
 *     does not wait, so it can be recorded into a CUDA graph with the rest;
 *   - a host pointer: copied back, and the call waits for the stream.  A
 *     capturing stream cannot wait, so while `stream` is being captured a
 *     host sum_plogp is refused with status 1 before any work is enqueued
 *     (the capture stays valid); pass NULL or a device pointer there.
 * The first call on a device looks up the array's device address and keeps
 * it for the life of the process; make that first call before any stream
 * capture, and make no call on a device after cudaDeviceReset of it (the
 * kept address would belong to the destroyed context).  All calls share the
 * one array: calls that overlap on the GPU (other streams, other host
 * threads) race.
 * Returns 0 on success, 1 for invalid or too large sizes (or a host
 * sum_plogp during capture), 2 for a CUDA error. */
int cuda_normalize_responsabilities_noalloc(real *d_respons, int N_slices, int N_images,
                                            void *stream, double *sum_plogp);

/* Status of the last call made through this header on the calling thread
 * (0 = success).  The reference reports errors only by printf
 * (emc_cuda.cu:178-181); this adds a way to read them. */
int emc_legacy_last_status(void);

#ifdef __cplusplus
}
#endif
