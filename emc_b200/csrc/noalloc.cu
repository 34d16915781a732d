// Responsibility normalisation that allocates nothing.
//
// Same kernels as cuda_normalize_responsabilities + cuda_total_respons, but
// their scratch -- one FP64 partial of sum P log P per block of 32 patterns,
// plus the final sum -- lives in a fixed array in device memory that is part
// of the library image, instead of buffers the library would cudaMalloc.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/emc.h"
#include "kernels.cuh"

namespace {

// Scratch limit: one partial per 32 patterns, so at most
// kMaxPartials * 32 = 2,097,152 patterns per call.  512 KB (+64 bytes) of
// device memory on every GPU that loads the library, held until exit.
constexpr int64_t kMaxPartials = 65536;
constexpr int64_t kPatternsPerPartial = 32;
__device__ __align__(256) double g_noalloc_scratch[kMaxPartials + 8];

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

// Device address of the scratch array for the current device.  In host code
// g_noalloc_scratch names a host-side stand-in, not device memory, so the
// address is looked up once per device with that device current and kept for
// the life of the process (a cudaDeviceReset of that device would leave it
// pointing into the destroyed context: the header forbids calls after one).
int scratch_for_current_device(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 2;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return 2;
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return 0;
}

}  // namespace

extern "C" int cuda_normalize_responsabilities_noalloc(real* d_respons, int N_slices,
                                                       int N_images, void* stream,
                                                       double* sum_plogp) {
  if (!d_respons || N_slices < 1 || N_images < 1) return 1;
  if ((int64_t)N_images > kMaxPartials * kPatternsPerPartial) return 1;  // scratch too small
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // where the sum goes: device (or managed) memory receives it on the stream;
  // host memory needs a copy and a wait, which a capturing stream cannot take
  bool sum_on_device = false;
  if (sum_plogp) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, sum_plogp) != cudaSuccess) {
      cudaGetLastError();
      return 1;
    }
    sum_on_device = attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
    if (!sum_on_device) {
      cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return 2;
      if (cap != cudaStreamCaptureStatusNone) return 1;  // refused before any stream work
    }
  }
  double* scratch = nullptr;
  if (scratch_for_current_device(&scratch) != 0) return 2;
  // every partial the sum reads is written by this call's softmax launch, so
  // nothing left in the array by an earlier call is read
  int nparts = 0;
  cudaError_t e = emc::launch_softmax_fp32(d_respons, N_slices, N_images, scratch, &nparts,
                                           nullptr, st);
  if (e == cudaSuccess)
    e = emc::launch_sum_f64(scratch, nparts, sum_on_device ? sum_plogp : scratch + kMaxPartials,
                            st);
  if (e == cudaSuccess && sum_plogp && !sum_on_device) {
    e = cudaMemcpyAsync(sum_plogp, scratch + kMaxPartials, sizeof(double),
                        cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  return e == cudaSuccess ? 0 : 2;
}
