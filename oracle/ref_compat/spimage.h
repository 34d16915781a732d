/*
 * Stand-in for the few libspimage declarations that the reference's emc.c
 * needs in order to compile.  It lets oracle/Makefile build the reference's
 * own CPU path functions (rotation sampling, detector coordinates, get_slice,
 * insert_slice, update_slice, slice_weighting, the likelihood functions) as
 * a test library under oracle/_ref/.  TEST INFRASTRUCTURE ONLY.
 *
 * Storage follows libspimage's column-major convention, which is also what
 * the reference's CUDA kernels assume when they index the uploaded arrays
 * directly (emc_cuda.cu:67 x_coordinates[y*x_max+x]; emc_cuda.cu:92
 * model[z*x*y + y*x + x]):
 *   sp_matrix  element (row, col) -> data[col*rows + row]
 *   sp_3matrix element (x, y, z)  -> data[z*x*y + y*x + x]
 * Functions that only the reference's main() uses (HDF5 image I/O, GSL,
 * allocation) are declared weak and left undefined: main() is renamed at
 * build time and never called.
 */
#pragma once
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

typedef float real;
typedef struct { real re, im; } Complex;

typedef struct { unsigned int rows, cols; real *data; } sp_matrix;
typedef struct { unsigned int rows, cols; int *data; } sp_imatrix;
typedef struct { unsigned int x, y, z; real *data; } sp_3matrix;
typedef struct { unsigned int x, y, z; Complex *data; } sp_c3matrix;
typedef struct { unsigned int x, y, z; int *data; } sp_i3matrix;
typedef struct { sp_c3matrix *image; sp_i3matrix *mask; } Image;

static inline unsigned int sp_matrix_rows(const sp_matrix *m) { return m->rows; }
static inline unsigned int sp_matrix_cols(const sp_matrix *m) { return m->cols; }
static inline unsigned int sp_matrix_size(const sp_matrix *m) { return m->rows * m->cols; }
static inline real sp_matrix_get(const sp_matrix *m, int r, int c) { return m->data[c * m->rows + r]; }
static inline void sp_matrix_set(sp_matrix *m, int r, int c, real v) { m->data[c * m->rows + r] = v; }
static inline unsigned int sp_imatrix_size(const sp_imatrix *m) { return m->rows * m->cols; }
static inline int sp_imatrix_get(const sp_imatrix *m, int r, int c) { return m->data[c * m->rows + r]; }
static inline void sp_imatrix_set(sp_imatrix *m, int r, int c, int v) { m->data[c * m->rows + r] = v; }
static inline unsigned int sp_3matrix_x(const sp_3matrix *m) { return m->x; }
static inline unsigned int sp_3matrix_y(const sp_3matrix *m) { return m->y; }
static inline unsigned int sp_3matrix_z(const sp_3matrix *m) { return m->z; }
static inline unsigned int sp_3matrix_size(const sp_3matrix *m) { return m->x * m->y * m->z; }
static inline real sp_3matrix_get(const sp_3matrix *m, int x, int y, int z) {
  return m->data[z * m->x * m->y + y * m->x + x];
}
static inline void sp_3matrix_set(sp_3matrix *m, int x, int y, int z, real v) {
  m->data[z * m->x * m->y + y * m->x + x] = v;
}
static inline real sp_min(real a, real b) { return a < b ? a : b; }
static inline real sp_cabs(Complex c) { return sqrtf(c.re * c.re + c.im * c.im); }
static inline Complex sp_cinit(real re, real im) { Complex c = {re, im}; return c; }

/* used only by the reference's main(); never called here */
__attribute__((weak)) sp_matrix *sp_matrix_alloc(unsigned int rows, unsigned int cols);
__attribute__((weak)) sp_imatrix *sp_imatrix_alloc(unsigned int rows, unsigned int cols);
__attribute__((weak)) sp_3matrix *sp_3matrix_alloc(unsigned int x, unsigned int y, unsigned int z);
__attribute__((weak)) Image *sp_image_read(const char *file, int flags);
__attribute__((weak)) void sp_image_write(Image *img, const char *file, int flags);
__attribute__((weak)) Image *sp_image_alloc(int x, int y, int z);
__attribute__((weak)) void sp_image_free(Image *img);
__attribute__((weak)) Image *sp_gaussian_blur(Image *img, real radius);
__attribute__((weak)) Complex sp_image_get(Image *img, int x, int y, int z);
__attribute__((weak)) int sp_image_x(Image *img);
__attribute__((weak)) int sp_image_y(Image *img);
__attribute__((weak)) int sp_image_z(Image *img);
/* the reference's CUDA wrappers, called only from main() */
#pragma weak cuda_update_slices
#pragma weak cuda_update_scaling
#pragma weak cuda_calculate_responsabilities
#pragma weak cuda_get_slices
#pragma weak cuda_allocate_slices
#pragma weak cuda_model_max
#pragma weak cuda_allocate_model
#pragma weak cuda_allocate_mask
#pragma weak cuda_reset_model
#pragma weak cuda_normalize_model
#pragma weak cuda_allocate_rotations
#pragma weak cuda_allocate_images
#pragma weak cuda_allocate_coords
#pragma weak cuda_allocate_real
#pragma weak cuda_allocate_scaling
#pragma weak cuda_normalize_responsabilities
#pragma weak cuda_total_respons
