// Register-tiled FP32-accumulate contraction used by the CUDA-core paths
// (plain FP32 EMC stages, the grouped candidate stages of the learned
// proposal, and the proposal network's layers).
#pragma once
#include <cstdint>
#include <type_traits>

namespace emc {

constexpr int kTileThreads = 256;

// C-tile of 128 rows x 64 columns per block (blockIdx.y, blockIdx.x), K-steps
// of 32, 256 threads with an 8x4 register tile each.  Op supplies the operand
// loads (a(row, k), b(col, k)), the per-element update, the epilogue, and may
// read blockIdx.z (grouped contractions).  The K extent comes from
// op.ksize() and may be 0 for an empty group.  An Op with a member
// origin(m0, n0) places its blocks itself (a list of tiles of uneven groups,
// indexed by blockIdx.x); a block whose origin() returns false exits.
constexpr int TM = 128, TN = 64, TK = 32;

template <class Op, class = void>
struct has_origin : std::false_type {};
template <class Op>
struct has_origin<Op, std::void_t<decltype(&Op::origin)>> : std::true_type {};

template <class Op>
__global__ void __launch_bounds__(kTileThreads) tile_kernel(const Op op) {
  __shared__ __align__(16) float As[TK][TM + 4];
  __shared__ __align__(16) float Bs[TK][TN + 4];
  const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
  int64_t m0, n0;
  if constexpr (has_origin<Op>::value) {
    if (!op.origin(m0, n0)) return;  // uniform over the block
  } else {
    m0 = (int64_t)blockIdx.y * TM;
    n0 = (int64_t)blockIdx.x * TN;
  }
  using Acc = typename Op::Acc;
  Acc acc[8][4];
  float tacc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      acc[i][j] = 0;
      tacc[i][j] = 0.0f;
    }
  float ra[16], rb[8];
  auto load = [&](int64_t k0) {
#pragma unroll
    for (int i = 0; i < 16; ++i) ra[i] = op.a(m0 + (t >> 5) + 8 * i, k0 + (t & 31));
    if constexpr (Op::kBKMajor) {
#pragma unroll
      for (int i = 0; i < 8; ++i) rb[i] = op.b(n0 + (t >> 5) + 8 * i, k0 + (t & 31));
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) rb[i] = op.b(n0 + (t & 63), k0 + (t >> 6) + 4 * i);
    }
  };
  auto stash = [&]() {
#pragma unroll
    for (int i = 0; i < 16; ++i) As[t & 31][(t >> 5) + 8 * i] = ra[i];
    if constexpr (Op::kBKMajor) {
#pragma unroll
      for (int i = 0; i < 8; ++i) Bs[t & 31][(t >> 5) + 8 * i] = rb[i];
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) Bs[(t >> 6) + 4 * i][t & 63] = rb[i];
    }
  };
  const int64_t K = op.ksize();
  load(0);
  for (int64_t k0 = 0; k0 < K; k0 += TK) {
    __syncthreads();
    stash();
    __syncthreads();
    if (k0 + TK < K) load(k0 + TK);
#pragma unroll 8
    for (int kk = 0; kk < TK; ++kk) {
      const float4 a0 = *reinterpret_cast<const float4*>(&As[kk][ty * 8]);
      const float4 a1 = *reinterpret_cast<const float4*>(&As[kk][ty * 8 + 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&Bs[kk][tx * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bv[4] = {b0.x, b0.y, b0.z, b0.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) tacc[i][j] = Op::inner(tacc[i][j], av[i], bv[j]);
    }
    // fold each 32-step partial into the (possibly FP64) running sum
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        acc[i][j] += (Acc)tacc[i][j];
        tacc[i][j] = 0.0f;
      }
  }
  __syncthreads();  // the epilogue may reuse As
  op.epilogue(acc, m0 + ty * 8, n0 + tx * 4, (float*)&As[0][0]);
}


}  // namespace emc
