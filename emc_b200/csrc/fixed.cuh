// Order-independent insertion: non-negative FP32 contributions summed exactly
// as fixed-point integers.
//
// A value x >= 0 is taken as the integer X = floor(x * 2^64) (64 fraction
// bits; x below 2^-64 contributes its bits above that point only) and added
// in 32-bit pieces to four 64-bit limbs, L_k += (X >> 32k) & (2^32 - 1).  An
// FP32 x has 24 significant bits, so it touches at most two neighbouring
// limbs; a limb overflows only after 2^32 additions.  Integer addition is
// associative, so the limbs after any set of additions do not depend on
// their order: sum = sum_k L_k 2^(32k - 64), rounded once to FP64 by
// fixed_value.  Per voxel 8 limbs: the insertion value (0..3) and its
// weight (4..7).
#pragma once
#include <cstdint>

namespace emc {

constexpr int kFixedLimbs = 4;

__device__ __forceinline__ void add_fixed(unsigned long long* L, float x) {
  if (!(x > 0.0f)) return;
  const uint32_t bits = __float_as_uint(x);
  const int ex = (int)((bits >> 23) & 0xffu);
  uint64_t m = bits & 0x7fffffu;
  // x = m 2^(ex - 150) for normal numbers (implicit bit added), m 2^-149 else;
  // b = position of m's lowest bit in X
  int b;
  if (ex == 0) {
    b = -149 + 64;
  } else {
    m |= 0x800000u;
    b = ex - 150 + 64;
  }
  if (b < 0) {
    if (b <= -24) return;
    m >>= -b;
    b = 0;
  }
  const int k = b >> 5;
  if (k >= kFixedLimbs) return;  // x >= 2^64: outside the format (not reached)
  const uint64_t v = m << (b & 31);  // < 2^55
  const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
  if (lo) atomicAdd(L + k, (unsigned long long)lo);
  if (hi && k + 1 < kFixedLimbs) atomicAdd(L + k + 1, (unsigned long long)hi);
}

__device__ __forceinline__ double fixed_value(const unsigned long long* L) {
  // highest limb first: every term is rounded to FP64 in the same order
  double s = (double)L[3] * 0x1p32;
  s = (s + (double)L[2]) * 0x1p32;
  s = (s + (double)L[1]) * 0x1p32;
  s = s + (double)L[0];
  return s * 0x1p-64;
}

}  // namespace emc
