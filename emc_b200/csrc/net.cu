// Orientation-proposal network: three 3x3 stride-2 convolutions (pad 1, ReLU)
// and a fully connected layer, softmax over the coarse rotations.  Input: one
// channel, in_side x in_side (the 2x-downsampled log(1+K) of a pattern).
//
// Layout: activations are channel-major across the batch, [C][B][H][W], so
// every layer is one contraction: im2col (col[ci*9+ky*3+kx][b*Ho*Wo+y*Wo+x])
// then out[co][n] = relu(W[co][k] col[k][n] + bias[co]).  Storage type T is
// __nv_bfloat16 (the network's precision) or float (gradient checks);
// contractions accumulate in FP32 (tile.cuh).  Parameters are one FP32 master
// array [W1 b1 W2 b2 W3 b3 Wfc bfc] with a T copy for the forward pass; Adam
// updates the master and refreshes the copy.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/emc_b200.h"
#include "tile.cuh"

namespace emc {
namespace {

template <class T>
__device__ __forceinline__ float ld(const T* p) {
  if constexpr (sizeof(T) == 2)
    return __bfloat162float(*p);
  else
    return *p;
}
template <class T>
__device__ __forceinline__ void st(T* p, float v) {
  if constexpr (sizeof(T) == 2)
    *p = __float2bfloat16_rn(v);
  else
    *p = v;
}

// C[r*scr + n*scn] (+)= sum_k A[r*sar + k*sak] B[n*sbn + k*sbk] (+ bias[r]) (relu)
// With kchunk > 0 the reduction is split: block z sums k in
// [z*kchunk, (z+1)*kchunk) and adds its partial into C atomically (C float,
// zeroed by the caller) -- the weight gradients, whose reduction runs over
// every output position of the batch.
template <class TA, class TB, class TC, bool BKMAJOR>
struct GemmOp {
  using Acc = float;
  static constexpr bool kBKMajor = BKMAJOR;
  const TA* A;
  const TB* B;
  TC* C;
  int64_t M, N, K, sar, sak, sbn, sbk, scr, scn;
  const float* bias;
  int relu, accumulate;
  int64_t kchunk;
  __device__ int64_t koff() const { return kchunk ? (int64_t)blockIdx.z * kchunk : 0; }
  __device__ int64_t ksize() const {
    if (!kchunk) return K;
    const int64_t left = K - koff();
    return left < kchunk ? left : kchunk;
  }
  __device__ float a(int64_t r, int64_t k) const {
    k += koff();
    return (r < M && k < K) ? ld(A + r * sar + k * sak) : 0.0f;
  }
  __device__ float b(int64_t n, int64_t k) const {
    k += koff();
    return (n < N && k < K) ? ld(B + n * sbn + k * sbk) : 0.0f;
  }
  static __device__ __forceinline__ float inner(float acc, float a, float b) { return fmaf(a, b, acc); }
  __device__ void epilogue(float (&acc)[8][4], int64_t r0, int64_t n0, float*) const {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int64_t r = r0 + i;
      if (r >= M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t n = n0 + j;
        if (n >= N) continue;
        TC* c = C + r * scr + n * scn;
        if constexpr (sizeof(TC) == 4) {
          if (kchunk) {
            atomicAdd(c, acc[i][j]);
            continue;
          }
        }
        float v = acc[i][j] + (bias ? bias[r] : 0.0f);
        if (accumulate) v += ld(c);
        if (relu) v = fmaxf(v, 0.0f);
        st(c, v);
      }
    }
  }
};

template <class TA, class TB, class TC, bool BKMAJOR>
cudaError_t gemm(const TA* A, int64_t sar, int64_t sak, const TB* B, int64_t sbn, int64_t sbk,
                 TC* C, int64_t scr, int64_t scn, int64_t M, int64_t N, int64_t K,
                 const float* bias, int relu, int accumulate, cudaStream_t st) {
  GemmOp<TA, TB, TC, BKMAJOR> op{A, B, C, M, N, K, sar, sak, sbn, sbk, scr, scn, bias, relu,
                                 accumulate, 0};
  dim3 grid((unsigned)((N + TN - 1) / TN), (unsigned)((M + TM - 1) / TM));
  tile_kernel<<<grid, kTileThreads, 0, st>>>(op);
  return cudaGetLastError();
}

// C[M][N] (row stride scr) = A B^T with the reduction split over enough
// blocks to fill the GPU (about 4 per SM); C is zeroed here.
template <class TA, class TB, bool BKMAJOR>
cudaError_t gemm_splitk(const TA* A, int64_t sar, int64_t sak, const TB* B, int64_t sbn,
                        int64_t sbk, float* C, int64_t scr, int64_t M, int64_t N, int64_t K,
                        int num_sms, cudaStream_t st) {
  const int64_t base = ((N + TN - 1) / TN) * ((M + TM - 1) / TM);
  int64_t splits = (4 * (int64_t)num_sms + base - 1) / base;
  const int64_t max_splits = (K + 255) / 256;  // at least 256 terms per block
  if (splits > max_splits) splits = max_splits;
  if (splits < 1) splits = 1;
  int64_t chunk = (K + splits - 1) / splits;
  chunk = (chunk + TK - 1) / TK * TK;
  splits = (K + chunk - 1) / chunk;
  cudaError_t e = cudaMemsetAsync(C, 0, sizeof(float) * M * scr, st);
  if (e != cudaSuccess) return e;
  GemmOp<TA, TB, float, BKMAJOR> op{A, B, C, M, N, K, sar, sak, sbn, sbk, scr, 1, nullptr, 0, 0,
                                    chunk};
  dim3 grid((unsigned)((N + TN - 1) / TN), (unsigned)((M + TM - 1) / TM), (unsigned)splits);
  tile_kernel<<<grid, kTileThreads, 0, st>>>(op);
  return cudaGetLastError();
}

template <class T>
__global__ void im2col_kernel(const T* in, int64_t B, int Cin, int H, T* col) {
  const int Ho = H / 2;
  const int64_t NN = B * Ho * Ho;
  const int64_t total = (int64_t)Cin * 9 * NN;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e / NN, n = e - k * NN;
    const int ci = (int)(k / 9), kk = (int)(k % 9), ky = kk / 3, kx = kk % 3;
    const int64_t b = n / (Ho * Ho);
    const int pos = (int)(n - b * Ho * Ho), y = pos / Ho, x = pos % Ho;
    const int yi = 2 * y + ky - 1, xi = 2 * x + kx - 1;
    float v = 0.0f;
    if (yi >= 0 && yi < H && xi >= 0 && xi < H) v = ld(in + (((int64_t)ci * B + b) * H + yi) * H + xi);
    st(col + e, v);
  }
}

// din[ci][b][yi][xi] = sum of dcol over the (ky, kx, y, x) with 2y+ky-1 = yi, 2x+kx-1 = xi
__global__ void col2im_kernel(const float* dcol, int64_t B, int Cin, int H, float* din) {
  const int Ho = H / 2;
  const int64_t NN = B * Ho * Ho;
  const int64_t total = (int64_t)Cin * B * H * H;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int xi = (int)(e % H), yi = (int)((e / H) % H);
    const int64_t b = (e / ((int64_t)H * H)) % B;
    const int ci = (int)(e / ((int64_t)H * H * B));
    float s = 0.0f;
    for (int ky = 0; ky < 3; ++ky) {
      const int ty = yi + 1 - ky;
      if (ty < 0 || (ty & 1) || ty / 2 >= Ho) continue;
      for (int kx = 0; kx < 3; ++kx) {
        const int tx = xi + 1 - kx;
        if (tx < 0 || (tx & 1) || tx / 2 >= Ho) continue;
        s += dcol[((int64_t)ci * 9 + ky * 3 + kx) * NN + b * Ho * Ho + (ty / 2) * Ho + tx / 2];
      }
    }
    din[e] = s;
  }
}

// feat[f][b] = out3[co][b*HW + pos] with f = co*HW + pos (and back)
template <class T>
__global__ void flatten_kernel(const T* out3, int64_t B, int C3, int HW, T* feat, int reverse,
                               const float* dfeat, float* dout3) {
  const int64_t total = (int64_t)C3 * HW * B;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = e / B, b = e - f * B;
    const int64_t co = f / HW, pos = f - co * HW;
    const int64_t o = (co * B + b) * HW + pos;
    if (!reverse)
      feat[e] = out3[o];
    else
      dout3[o] = dfeat[e];
  }
}

// per column b: softmax over C of z[c][b]; probs[b][c]; with targets t[b][c]:
// loss (sum over the batch of -sum_c t log softmax) and dz[c][b] = (p - t) / B
__global__ void softmax_xent_kernel(const float* z, int64_t B, int C, const float* t, float* probs,
                                    float* dz, double* loss) {
  const int64_t b = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (b >= B) return;
  float mx = -INFINITY;
  for (int c = lane; c < C; c += 32) mx = fmaxf(mx, z[(int64_t)c * B + b]);
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  float s = 0.0f;
  for (int c = lane; c < C; c += 32) s += expf(z[(int64_t)c * B + b] - mx);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const float lse = mx + logf(s);
  double l = 0.0;
  for (int c = lane; c < C; c += 32) {
    const float zc = z[(int64_t)c * B + b];
    const float p = expf(zc - lse);
    if (probs) probs[b * C + c] = p;
    if (t) {
      const float tc = t[b * C + c];
      if (tc > 0.0f) l -= (double)tc * (double)(zc - lse);
      dz[(int64_t)c * B + b] = (p - tc) / (float)B;
    }
  }
  if (t) {
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if (lane == 0) atomicAdd(loss, l);
  }
}

template <class T>
__global__ void relu_back_kernel(float* d, const T* out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (!(ld(out + i) > 0.0f)) d[i] = 0.0f;
}

// db[r] = sum_n d[r][n]
__global__ void rowsum_grad_kernel(const float* d, int64_t rows, int64_t n, float* db) {
  const int64_t r = blockIdx.x;
  float s = 0.0f;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) s += d[r * n + i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ float red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    db[r] = t;
  }
  (void)rows;
}

template <class T>
__global__ void adam_kernel(float* w, T* wc, const float* g, float* m, float* v, int64_t n,
                            float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    st(wc + i, wi);
  }
}

template <class T>
__global__ void copy_params_kernel(const float* w, T* wc, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    st(wc + i, w[i]);
}

inline unsigned blocks_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (unsigned)(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

}  // namespace
}  // namespace emc

using namespace emc;

struct emc_net {
  int S = 0, C = 0, bf16 = 1, num_sms = 148;
  int ch[4] = {1, 16, 32, 64};
  int64_t off[9] = {0};  // parameter offsets: W1 b1 W2 b2 W3 b3 Wfc bfc, total
  int64_t F = 0, cap = 0;  // fc input features, batch capacity
  int64_t step = 0;
  float* w = nullptr;   // FP32 master
  void* wc = nullptr;   // T copy
  float* g = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  // activations (T) and gradients (float)
  void *col[3] = {nullptr}, *out[3] = {nullptr}, *feat = nullptr;
  float *z = nullptr, *dz = nullptr, *dfeat = nullptr, *dout[3] = {nullptr};
  float* dcol = nullptr;
  double* d_loss = nullptr;
  cudaStream_t st = nullptr;
  std::vector<void*> bufs;
  std::string err;

  int side(int l) const { return S >> l; }  // input side of layer l (0..3)
  size_t tsz() const { return bf16 ? 2 : 4; }
  emc_status fail(cudaError_t e, const char* what) {
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? EMC_ERR_OOM : EMC_ERR_CUDA;
  }
  void* dalloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) return nullptr;
    bufs.push_back(p);
    return p;
  }
  void release_batch() {
    // frees the batch-sized buffers (everything after the 5 parameter arrays)
    for (size_t i = 5; i < bufs.size(); ++i) cudaFree(bufs[i]);
    if (bufs.size() > 5) bufs.resize(5);
  }
  bool ensure(int64_t B) {
    if (B <= cap) return true;
    release_batch();
    for (int l = 0; l < 3; ++l) {
      const int64_t NN = B * (int64_t)side(l + 1) * side(l + 1);
      if (!(col[l] = dalloc(tsz() * ch[l] * 9 * NN)) || !(out[l] = dalloc(tsz() * ch[l + 1] * NN)) ||
          !(dout[l] = (float*)dalloc(4 * ch[l + 1] * NN)))
        return false;
    }
    // dcol holds the layer-1 input columns in the forward pass (9 x NN1) and
    // the column gradients of layers 2 and 3 in the backward pass
    int64_t dcol_n = 9 * B * (int64_t)side(1) * side(1);
    for (int l = 1; l < 3; ++l) {
      const int64_t k = (int64_t)ch[l] * 9 * B * side(l + 1) * side(l + 1);
      if (k > dcol_n) dcol_n = k;
    }
    if (!(feat = dalloc(tsz() * F * B)) || !(z = (float*)dalloc(4 * C * B)) ||
        !(dz = (float*)dalloc(4 * C * B)) || !(dfeat = (float*)dalloc(4 * F * B)) ||
        !(dcol = (float*)dalloc(4 * dcol_n)))
      return false;
    cap = B;
    return true;
  }
};

namespace {

template <class T>
cudaError_t net_forward(emc_net* n, const float* x, int64_t B, float* probs, const float* t) {
  cudaStream_t st = n->st;
  const T* wc = static_cast<const T*>(n->wc);
  cudaError_t e = cudaSuccess;
  for (int l = 0; l < 3 && e == cudaSuccess; ++l) {
    const int H = n->side(l), Ho = n->side(l + 1);
    const int64_t NN = B * (int64_t)Ho * Ho;
    const int64_t K9 = (int64_t)n->ch[l] * 9;
    if (l == 0) {
      // layer 1 reads the FP32 input directly (one channel, [B][S][S])
      im2col_kernel<float><<<blocks_for(K9 * NN), 256, 0, st>>>(x, B, 1, H, n->dcol);
      // the FP32 column buffer (dcol is free during the forward pass) into T
      copy_params_kernel<T><<<blocks_for(K9 * NN), 256, 0, st>>>(n->dcol, (T*)n->col[0], K9 * NN);
    } else {
      im2col_kernel<T><<<blocks_for(K9 * NN), 256, 0, st>>>((const T*)n->out[l - 1], B, n->ch[l], H,
                                                            (T*)n->col[l]);
    }
    // out[co][n] = relu(W[co][k] col[k][n] + b[co])
    e = gemm<T, T, T, false>(wc + n->off[2 * l], K9, 1, (const T*)n->col[l], 1, NN,
                             (T*)n->out[l], NN, 1, n->ch[l + 1], NN, K9, n->w + n->off[2 * l + 1], 1,
                             0, st);
  }
  if (e != cudaSuccess) return e;
  const int HW3 = n->side(3) * n->side(3);
  flatten_kernel<T><<<blocks_for(n->F * B), 256, 0, st>>>((const T*)n->out[2], B, n->ch[3], HW3,
                                                          (T*)n->feat, 0, nullptr, nullptr);
  // z[c][b] = Wfc[c][f] feat[f][b] + bfc[c]
  e = gemm<T, T, float, false>(wc + n->off[6], n->F, 1, (const T*)n->feat, 1, B, n->z, B, 1, n->C, B,
                               n->F, n->w + n->off[7], 0, 0, st);
  if (e != cudaSuccess) return e;
  if (t) {
    e = cudaMemsetAsync(n->d_loss, 0, sizeof(double), st);
    if (e != cudaSuccess) return e;
  }
  softmax_xent_kernel<<<(unsigned)((B + 7) / 8), 256, 0, st>>>(n->z, B, n->C, t, probs, n->dz,
                                                               n->d_loss);
  return cudaGetLastError();
}

template <class T>
cudaError_t net_backward(emc_net* n, int64_t B) {
  cudaStream_t st = n->st;
  const T* wc = static_cast<const T*>(n->wc);
  float* g = n->g;
  cudaError_t e;
  // fc: dWfc[c][f] = dz[c][b] feat[f][b];  dbfc = sum_b dz;  dfeat[f][b] = Wfc[c][f] dz[c][b]
  e = gemm_splitk<float, T, true>(n->dz, B, 1, (const T*)n->feat, B, 1, g + n->off[6], n->F, n->C,
                                  n->F, B, n->num_sms, st);
  if (e != cudaSuccess) return e;
  rowsum_grad_kernel<<<(unsigned)n->C, 256, 0, st>>>(n->dz, n->C, B, g + n->off[7]);
  e = gemm<T, float, float, false>(wc + n->off[6], 1, n->F, n->dz, 1, B, n->dfeat, B, 1, n->F, B,
                                   n->C, nullptr, 0, 0, st);
  if (e != cudaSuccess) return e;
  const int HW3 = n->side(3) * n->side(3);
  flatten_kernel<T><<<blocks_for(n->F * B), 256, 0, st>>>(nullptr, B, n->ch[3], HW3, nullptr, 1,
                                                          n->dfeat, n->dout[2]);
  for (int l = 2; l >= 0; --l) {
    const int H = n->side(l), Ho = n->side(l + 1);
    const int64_t NN = B * (int64_t)Ho * Ho;
    const int64_t K9 = (int64_t)n->ch[l] * 9;
    const int64_t cout = n->ch[l + 1];
    relu_back_kernel<T><<<blocks_for(cout * NN), 256, 0, st>>>(n->dout[l], (const T*)n->out[l],
                                                               cout * NN);
    // dW[co][k] = dout[co][n] col[k][n];  db[co] = sum_n dout[co][n]
    e = gemm_splitk<float, T, true>(n->dout[l], NN, 1, (const T*)n->col[l], NN, 1,
                                    g + n->off[2 * l], K9, cout, K9, NN, n->num_sms, st);
    if (e != cudaSuccess) return e;
    rowsum_grad_kernel<<<(unsigned)cout, 256, 0, st>>>(n->dout[l], cout, NN, g + n->off[2 * l + 1]);
    if (l == 0) break;
    // dcol[k][n] = W[co][k] dout[co][n];  then col2im into the previous layer's dout
    e = gemm<T, float, float, false>(wc + n->off[2 * l], 1, K9, n->dout[l], 1, NN, n->dcol, NN, 1,
                                     K9, NN, cout, nullptr, 0, 0, st);
    if (e != cudaSuccess) return e;
    col2im_kernel<<<blocks_for((int64_t)n->ch[l] * B * H * H), 256, 0, st>>>(n->dcol, B, n->ch[l], H,
                                                                            n->dout[l - 1]);
  }
  return cudaGetLastError();
}

}  // namespace

extern "C" {

emc_status emc_net_create(int in_side, int n_out, int bf16, uint64_t seed, int device,
                          emc_net** out) {
  if (!out || in_side < 8 || (in_side % 8) || n_out < 2) return EMC_ERR_ARG;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return EMC_ERR_CUDA;
  emc_net* n = new emc_net();
  cudaDeviceGetAttribute(&n->num_sms, cudaDevAttrMultiProcessorCount, device);
  n->S = in_side;
  n->C = n_out;
  n->bf16 = bf16 ? 1 : 0;
  n->F = (int64_t)n->ch[3] * n->side(3) * n->side(3);
  int64_t o = 0;
  for (int l = 0; l < 3; ++l) {
    n->off[2 * l] = o;
    o += (int64_t)n->ch[l + 1] * n->ch[l] * 9;
    n->off[2 * l + 1] = o;
    o += n->ch[l + 1];
  }
  n->off[6] = o;
  o += (int64_t)n->C * n->F;
  n->off[7] = o;
  o += n->C;
  n->off[8] = o;
  // He-normal initialisation, biases 0
  std::vector<float> h(o, 0.0f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < 4; ++l) {
    const int64_t fan_in = l < 3 ? (int64_t)n->ch[l] * 9 : n->F;
    std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (float)fan_in) * (l < 3 ? 1.0f : 0.5f));
    for (int64_t i = n->off[2 * l]; i < n->off[2 * l + 1]; ++i) h[i] = nd(rng);
  }
  emc_status s = EMC_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&n->st, cudaStreamNonBlocking);
  if (e != cudaSuccess ||
      !(n->w = (float*)n->dalloc(4 * o)) || !(n->wc = n->dalloc(n->tsz() * o)) ||
      !(n->g = (float*)n->dalloc(4 * o)) || !(n->m = (float*)n->dalloc(4 * o)) ||
      !(n->v = (float*)n->dalloc(4 * o)))
    s = EMC_ERR_OOM;
  if (s == EMC_OK) {
    cudaMalloc(&n->d_loss, sizeof(double));
    cudaMemcpy(n->w, h.data(), 4 * o, cudaMemcpyHostToDevice);
    cudaMemset(n->m, 0, 4 * o);
    cudaMemset(n->v, 0, 4 * o);
    if (n->bf16)
      copy_params_kernel<__nv_bfloat16><<<blocks_for(o), 256, 0, n->st>>>(n->w, (__nv_bfloat16*)n->wc, o);
    else
      copy_params_kernel<float><<<blocks_for(o), 256, 0, n->st>>>(n->w, (float*)n->wc, o);
    if ((e = cudaStreamSynchronize(n->st)) != cudaSuccess) s = n->fail(e, "emc_net_create");
  }
  if (s != EMC_OK) {
    emc_net_destroy(n);
    return s;
  }
  *out = n;
  return EMC_OK;
}

emc_status emc_net_destroy(emc_net* n) {
  if (!n) return EMC_OK;
  if (n->st) cudaStreamSynchronize(n->st);
  for (void* p : n->bufs) cudaFree(p);
  if (n->d_loss) cudaFree(n->d_loss);
  if (n->st) cudaStreamDestroy(n->st);
  delete n;
  return EMC_OK;
}

int64_t emc_net_num_params(const emc_net* n) { return n ? n->off[8] : 0; }

emc_status emc_net_get_params(emc_net* n, float* host) {
  if (!n || !host) return EMC_ERR_ARG;
  cudaError_t e = cudaMemcpyAsync(host, n->w, 4 * n->off[8], cudaMemcpyDeviceToHost, n->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(n->st);
  return e == cudaSuccess ? EMC_OK : n->fail(e, "emc_net_get_params");
}

emc_status emc_net_set_params(emc_net* n, const float* host) {
  if (!n || !host) return EMC_ERR_ARG;
  const int64_t o = n->off[8];
  cudaError_t e = cudaMemcpyAsync(n->w, host, 4 * o, cudaMemcpyHostToDevice, n->st);
  if (e == cudaSuccess) {
    if (n->bf16)
      copy_params_kernel<__nv_bfloat16><<<blocks_for(o), 256, 0, n->st>>>(n->w, (__nv_bfloat16*)n->wc, o);
    else
      copy_params_kernel<float><<<blocks_for(o), 256, 0, n->st>>>(n->w, (float*)n->wc, o);
    e = cudaStreamSynchronize(n->st);
  }
  return e == cudaSuccess ? EMC_OK : n->fail(e, "emc_net_set_params");
}

emc_status emc_net_forward(emc_net* n, const float* x, int64_t batch, float* probs) {
  if (!n || !x || !probs || batch < 1) return EMC_ERR_ARG;
  if (!n->ensure(batch)) return EMC_ERR_OOM;
  cudaError_t e = n->bf16 ? net_forward<__nv_bfloat16>(n, x, batch, probs, nullptr)
                          : net_forward<float>(n, x, batch, probs, nullptr);
  if (e == cudaSuccess) e = cudaStreamSynchronize(n->st);
  return e == cudaSuccess ? EMC_OK : n->fail(e, "emc_net_forward");
}

emc_status emc_net_gradients(emc_net* n, const float* x, const float* t, int64_t batch,
                             double* loss, float* grad_host) {
  if (!n || !x || !t || batch < 1) return EMC_ERR_ARG;
  if (!n->ensure(batch)) return EMC_ERR_OOM;
  cudaError_t e = n->bf16 ? net_forward<__nv_bfloat16>(n, x, batch, nullptr, t)
                          : net_forward<float>(n, x, batch, nullptr, t);
  if (e == cudaSuccess)
    e = n->bf16 ? net_backward<__nv_bfloat16>(n, batch) : net_backward<float>(n, batch);
  double h = 0.0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, n->d_loss, sizeof(double), cudaMemcpyDeviceToHost, n->st);
  if (e == cudaSuccess && grad_host)
    e = cudaMemcpyAsync(grad_host, n->g, 4 * n->off[8], cudaMemcpyDeviceToHost, n->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(n->st);
  if (e != cudaSuccess) return n->fail(e, "emc_net_gradients");
  if (loss) *loss = h / (double)batch;
  return EMC_OK;
}

emc_status emc_net_train_step(emc_net* n, const float* x, const float* t, int64_t batch,
                              float lr, double* loss) {
  emc_status s = emc_net_gradients(n, x, t, batch, loss, nullptr);
  if (s != EMC_OK) return s;
  n->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
  const int64_t o = n->off[8];
  if (n->bf16)
    adam_kernel<__nv_bfloat16><<<blocks_for(o), 256, 0, n->st>>>(n->w, (__nv_bfloat16*)n->wc, n->g,
                                                                 n->m, n->v, o, lr, b1, b2, 1e-8f, c1, c2);
  else
    adam_kernel<float><<<blocks_for(o), 256, 0, n->st>>>(n->w, (float*)n->wc, n->g, n->m, n->v, o, lr,
                                                         b1, b2, 1e-8f, c1, c2);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? EMC_OK : n->fail(e, "emc_net_train_step");
}

const char* emc_net_last_error(const emc_net* n) { return n ? n->err.c_str() : ""; }

}  // extern "C"
