// Reference-compatible C API (include/emc.h): the cuda_* functions of
// FilipeMaia/emc emc_cuda.cu / emc_atomic.cu with the same names, arguments
// and synchronous behaviour, implemented on the engine's FP32 kernels.
// Like the reference, these functions share process-wide state (cached
// work buffers) and are not thread-safe.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/emc.h"
#include "kernels.cuh"

using namespace emc;

namespace {

thread_local int g_status = 0;

struct Work {
  // cached device buffers, grown on demand (the reference cudaMallocs per call)
  void* buf[8] = {nullptr};
  size_t cap[8] = {0};
  std::vector<int32_t> mask_host;
  int32_t* pix = nullptr;
  int64_t npa = 0;
  const int* pix_key = nullptr;
  int64_t pix_n = -1;

  template <class T>
  T* get(int slot, size_t count) {
    const size_t bytes = count * sizeof(T) + 16;
    if (cap[slot] < bytes) {
      if (buf[slot]) cudaFree(buf[slot]);
      buf[slot] = nullptr;
      cap[slot] = 0;
      if (cudaMalloc(&buf[slot], bytes) != cudaSuccess) return nullptr;
      cap[slot] = bytes;
    }
    return static_cast<T*>(buf[slot]);
  }
};
Work g;

bool ok(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return true;
  std::fprintf(stderr, "CUDA Error: %s (%s)\n", cudaGetErrorString(e), where);
  g_status = (int)e;
  return false;
}

// Active-pixel list (mask != 0) of a device mask, rebuilt when the mask changes.
int32_t* active_pixels(const int* d_mask, int64_t n, int64_t* npa) {
  std::vector<int32_t> m(n);
  if (!ok(cudaMemcpy(m.data(), d_mask, sizeof(int32_t) * n, cudaMemcpyDeviceToHost), "mask"))
    return nullptr;
  if (g.pix && g.pix_key == d_mask && g.pix_n == n && m == g.mask_host) {
    *npa = g.npa;
    return g.pix;
  }
  std::vector<int32_t> pix;
  for (int64_t i = 0; i < n; ++i)
    if (m[i] != 0) pix.push_back((int32_t)i);
  int32_t* d = g.get<int32_t>(0, pix.size() + 1);
  if (!d || !ok(cudaMemcpy(d, pix.data(), sizeof(int32_t) * pix.size(), cudaMemcpyHostToDevice),
                "pix"))
    return nullptr;
  g.mask_host.swap(m);
  g.pix = d;
  g.pix_key = d_mask;
  g.pix_n = n;
  g.npa = (int64_t)pix.size();
  *npa = g.npa;
  return d;
}

}  // namespace

extern "C" {

int emc_legacy_last_status(void) { return g_status; }

void cuda_allocate_slices(real** slices, Setup setup, int N_slices) {
  g_status = 0;
  ok(cudaMalloc(slices, sizeof(real) * (size_t)setup.side * setup.side * N_slices), "slices");
}

void cuda_allocate_model(real** d_model, sp_3matrix* model) {
  g_status = 0;
  const size_t n = (size_t)model->x * model->y * model->z;
  if (ok(cudaMalloc(d_model, sizeof(real) * n), "model"))
    ok(cudaMemcpy(*d_model, model->data, sizeof(real) * n, cudaMemcpyHostToDevice), "model");
}

void cuda_allocate_mask(int** d_mask, sp_imatrix* mask) {
  g_status = 0;
  const size_t n = (size_t)mask->rows * mask->cols;
  if (ok(cudaMalloc(d_mask, sizeof(int) * n), "mask"))
    ok(cudaMemcpy(*d_mask, mask->data, sizeof(int) * n, cudaMemcpyHostToDevice), "mask");
}

void cuda_allocate_rotations(real** d_rotations, Quaternion** rotations, int N_slices) {
  g_status = 0;
  std::vector<real> q(4 * (size_t)N_slices);
  for (int i = 0; i < N_slices; ++i) std::memcpy(&q[4 * (size_t)i], rotations[i]->q, 4 * sizeof(real));
  if (ok(cudaMalloc(d_rotations, sizeof(real) * q.size()), "rotations"))
    ok(cudaMemcpy(*d_rotations, q.data(), sizeof(real) * q.size(), cudaMemcpyHostToDevice), "rotations");
}

void cuda_allocate_images(real** d_images, sp_matrix** images, int N_images) {
  g_status = 0;
  const size_t n = (size_t)images[0]->rows * images[0]->cols;
  if (!ok(cudaMalloc(d_images, sizeof(real) * n * N_images), "images")) return;
  for (int i = 0; i < N_images; ++i)
    if (!ok(cudaMemcpy(*d_images + n * i, images[i]->data, sizeof(real) * n, cudaMemcpyHostToDevice),
            "images"))
      return;
}

void cuda_allocate_coords(real** d_x, real** d_y, real** d_z, sp_matrix* x, sp_matrix* y,
                          sp_matrix* z) {
  g_status = 0;
  const size_t n = (size_t)x->rows * x->cols;
  real** d[3] = {d_x, d_y, d_z};
  sp_matrix* h[3] = {x, y, z};
  for (int k = 0; k < 3; ++k) {
    if (!ok(cudaMalloc(d[k], sizeof(real) * n), "coords")) return;
    if (!ok(cudaMemcpy(*d[k], h[k]->data, sizeof(real) * n, cudaMemcpyHostToDevice), "coords")) return;
  }
}

void cuda_allocate_real(real** x, int n) {
  g_status = 0;
  ok(cudaMalloc(x, (size_t)n), "real");  // n is in bytes (emc_cuda.cu:435-437)
}

void cuda_allocate_scaling(real** d_scaling, int N_images) {
  g_status = 0;
  if (ok(cudaMalloc(d_scaling, sizeof(real) * N_images), "scaling"))
    ok(launch_fill(*d_scaling, N_images, 1.0f, 0), "scaling");
}

void cuda_reset_model(sp_3matrix* model, real* d_model) {
  g_status = 0;
  ok(cudaMemset(d_model, 0, sizeof(real) * (size_t)model->x * model->y * model->z), "reset");
}

void cuda_get_slices(sp_3matrix* model, real* d_model, real* d_slices, real* d_rot, real* d_x,
                     real* d_y, real* d_z, int N_slices) {
  g_status = 0;
  ExpandArgs a{};
  a.model = d_model;
  a.quat = d_rot;
  a.cx = d_x;
  a.cy = d_y;
  a.cz = d_z;
  a.R = N_slices;
  a.npix = (int64_t)model->x * model->y;  // slices have the model's x*y pixels (emc_cuda.cu:275-277)
  a.ld = a.npix;
  a.side = (int)model->x;
  a.interp = 0;
  a.out = EXP_F32;
  a.stat = STAT_NONE;
  a.out_f32 = d_slices;
  if (ok(launch_expand(a, 0), "get_slices")) ok(cudaDeviceSynchronize(), "get_slices");
}

void cuda_calculate_responsabilities(real* d_slices, real* d_images, int* d_mask, real sigma,
                                     real* d_scaling, real* d_respons, int N_2d, int N_images,
                                     int N_slices, real* respons) {
  g_status = 0;
  int64_t npa = 0;
  int32_t* pix = active_pixels(d_mask, N_2d, &npa);
  if (!pix) return;
  LLArgs l{};
  l.A = d_slices;
  l.K = d_images;
  l.pix = pix;
  l.scaling = d_scaling;
  l.R = N_slices;
  l.N = N_images;
  l.npa = npa;
  l.ldA = N_2d;
  l.ldK = N_2d;
  l.ldLL = N_images;
  l.gauss_inv = 1.0 / (2.0 * (double)npa * (double)sigma * (double)sigma);
  l.poisson = 0;
  l.LL = d_respons;
  if (!ok(launch_ll_fp32(l, 0), "responsabilities")) return;
  // emc_cuda.cu:182: the whole matrix is copied to the host array
  ok(cudaMemcpy(respons, d_respons, sizeof(real) * (size_t)N_slices * N_images,
                cudaMemcpyDeviceToHost),
     "respons");
}

void cuda_normalize_responsabilities(real* d_respons, int N_slices, int N_images) {
  g_status = 0;
  double* part = g.get<double>(1, (size_t)(N_images + 31) / 32 + 1);
  if (!part) {
    g_status = (int)cudaErrorMemoryAllocation;
    return;
  }
  int np = 0;
  ok(launch_softmax_fp32(d_respons, N_slices, N_images, part, &np, nullptr, 0),
     "normalize_responsabilities");
}

real cuda_total_respons(real* d_respons, real* respons, int n) {
  g_status = 0;
  (void)respons;
  double* scratch = g.get<double>(2, 1024);
  if (!scratch) return 0;
  if (!ok(launch_xlogx_sum(d_respons, n, scratch + 1000, scratch, 0), "total_respons")) return 0;
  double h = 0;
  ok(cudaMemcpy(&h, scratch + 1000, sizeof(double), cudaMemcpyDeviceToHost), "total_respons");
  return (real)h;
}

void cuda_update_scaling(real* d_images, real* d_slices, int* d_mask, real* d_respons,
                         real* d_scaling, int N_images, int N_slices, int N_2d, real* scaling) {
  g_status = 0;
  int64_t npa = 0;
  int32_t* pix = active_pixels(d_mask, N_2d, &npa);
  if (!pix) return;
  const int64_t nparts = ((int64_t)N_slices + 127) / 128;
  double* num = g.get<double>(3, (size_t)N_images);
  double* den = g.get<double>(4, (size_t)nparts * N_images);
  if (!num || !den) {
    g_status = (int)cudaErrorMemoryAllocation;
    return;
  }
  if (!ok(launch_pattern_stats(d_images, pix, N_images, npa, N_2d, 1, num, 0), "scaling")) return;
  CrossArgs x{};
  x.S = d_slices;
  x.K = d_images;
  x.pix = pix;
  x.P = d_respons;
  x.R = N_slices;
  x.N = N_images;
  x.npa = npa;
  x.ldS = N_2d;
  x.ldK = N_2d;
  x.den_part = den;
  if (!ok(launch_scaling_cross(x, 0), "scaling")) return;
  if (!ok(launch_scaling_finish(num, den, nparts, N_images, d_scaling, 0), "scaling")) return;
  ok(cudaMemcpy(scaling, d_scaling, sizeof(real) * N_images, cudaMemcpyDeviceToHost), "scaling");
}

real cuda_update_slices(real* d_images, real* d_slices, int* d_mask, real* d_respons,
                        real* d_scaling, int N_images, int N_slices, int N_2d, sp_3matrix* model,
                        real* d_model, real* d_x, real* d_y, real* d_z, real* d_rot,
                        real* weights, real* d_weight, Setup setup, sp_matrix** images) {
  g_status = 0;
  (void)setup;
  (void)images;
  int64_t npa = 0;
  int32_t* pix = active_pixels(d_mask, N_2d, &npa);
  if (!pix) return 0;
  float* T = g.get<float>(5, (size_t)N_slices);
  float* rotw = g.get<float>(6, (size_t)N_slices);
  if (!T || !rotw) {
    g_status = (int)cudaErrorMemoryAllocation;
    return 0;
  }
  if (!ok(cudaMemcpy(rotw, weights, sizeof(real) * N_slices, cudaMemcpyHostToDevice), "weights"))
    return 0;
  if (!ok(launch_row_sums(d_respons, N_slices, N_images, T, 0), "update_slices")) return 0;
  CompressArgs a{};
  a.P = d_respons;
  a.K = d_images;
  a.pix = pix;
  a.scaling = d_scaling;
  a.T = T;
  a.R = N_slices;
  a.N = N_images;
  a.npa = npa;
  a.ldK = N_2d;
  a.ldU = N_2d;
  a.U = d_slices;
  if (!ok(launch_compress_fp32(a, 0), "update_slices")) return 0;
  InsertArgs in{};
  in.U = d_slices;
  in.T = T;
  in.rotw = rotw;
  in.quat = d_rot;
  in.cx = d_x;
  in.cy = d_y;
  in.cz = d_z;
  in.ins = d_mask;
  in.R = N_slices;
  in.npix = N_2d;
  in.ldU = N_2d;
  in.side = (int)model->x;
  in.interp = 0;
  in.model = d_model;
  in.weight = d_weight;
  if (!ok(launch_insert(in, 0), "update_slices")) return 0;
  std::vector<float> t(N_slices);
  if (!ok(cudaMemcpy(t.data(), T, sizeof(float) * N_slices, cudaMemcpyDeviceToHost), "T")) return 0;
  real total = 0;
  for (float v : t) total += v;
  // emc_cuda.cu:352: the (not yet normalised) model is copied to the host
  ok(cudaMemcpy(model->data, d_model, sizeof(real) * (size_t)model->x * model->y * model->z,
                cudaMemcpyDeviceToHost),
     "model");
  return total;
}

void cuda_normalize_model(sp_3matrix* model, real* d_model, real* d_weight) {
  g_status = 0;
  double* scratch = g.get<double>(7, 1024);
  if (!scratch) return;
  if (ok(launch_normalize_model(d_model, d_weight, (int64_t)model->x * model->y * model->z, 0,
                                scratch, scratch + 1000, 0),
         "normalize_model"))
    ok(cudaDeviceSynchronize(), "normalize_model");
}

real cuda_model_max(real* model, int model_size) {
  g_status = 0;
  double* scratch = g.get<double>(2, 1024);
  if (!scratch) return 0;
  if (!ok(launch_model_max(model, model_size, scratch, scratch + 1000, 0), "model_max")) return 0;
  double h = 0;
  ok(cudaMemcpy(&h, scratch + 1000, sizeof(double), cudaMemcpyDeviceToHost), "model_max");
  // thrust::reduce with init 0 (emc_cuda.cu:366)
  return (real)(h > 0 ? h : 0);
}

}  // extern "C"
