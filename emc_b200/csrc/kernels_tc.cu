// Mixed-precision path for sm_100a: two tcgen05 contractions (TMA-fed shared
// memory operands, TMEM accumulators, warp-specialised persistent CTAs) and
// the FP64 responsibility pass between them.
//
//   maximize : acc[p][r] = sum_j K_pj (B_hi + B_lo)_rj      (B = log W or S)
//   compress : acc[r][j] = sum_p (P'_hi + P'_lo)_rp K_pj     (P' = c0 P / phi)
// Counts are integers <= 2048, exact in FP16; the other operand is split into
// an FP16 hi part and an FP16 remainder, so each k-step issues two MMAs into
// the same FP32 accumulator.
//
// CTA: 192 threads.  warp 0 = TMA producer, warp 1 = MMA issuer (and TMEM
// owner), warps 2-5 = epilogue (TMEM lane quarter = warp % 4).  Two 256-column
// FP32 accumulators in TMEM let the epilogue of tile i overlap the MMAs of
// tile i+1.  Every mbarrier wait is bounded; on expiry the kernel records the
// site in TcStatus, drains its copies and MMAs, frees TMEM and returns.
#include <cfloat>
#include <cstdint>

#include "tc.cuh"
#include "voxel.h"

namespace emc {
namespace {

constexpr int BM = 128, BN = 256, BK = 64;
constexpr int kThreads = 192;
constexpr int kTmemCols = 512;
constexpr uint64_t kWaitLimitNs = 10ull * 1000ull * 1000ull * 1000ull;
constexpr uint32_t A_BYTES = BM * BK * 2;  // 16 KB
constexpr uint32_t B_BYTES = BN * BK * 2;  // 32 KB

// ------------------------------------------------------------ PTX helpers --
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* tm, int c0, int c1,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)tm), "r"(c0), "r"(c1), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void mma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major operand, 128-byte swizzle, rows of
// 128 bytes, 8-row core groups 1024 bytes apart (SBO); LBO unused for this
// layout; version 1 (sm_100).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  uint64_t d = (uint64_t)((addr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
// Instruction descriptor, kind::f16: D = F32, A = B = F16, both K-major.
constexpr uint32_t kIdesc = (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(BN >> 3) << 17) |
                            ((uint32_t)(BM >> 4) << 24);

struct Ctl {
  volatile int* abort;
  TcStatus* st;
};

__device__ bool bounded_wait(uint32_t bar, uint32_t parity, const Ctl& c, int site) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_test(bar, parity)) return true;
    if ((it & 31) == 0) {
      if (*c.abort) return false;
      if (globaltimer() - t0 > kWaitLimitNs) {
        *c.abort = 1;
        if (atomicCAS(&c.st->code, 0, TC_TIMEOUT) == 0) {
          c.st->where = site;
          c.st->block = blockIdx.x;
        }
        return false;
      }
    }
  }
}

// ---------------------------------------------------------------- kernel --
template <int NA, int NB, int STAGES, bool M_INNER, class Epi>
__global__ void __launch_bounds__(kThreads, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA0, const __grid_constant__ CUtensorMap tmA1,
                   const __grid_constant__ CUtensorMap tmB0, const __grid_constant__ CUtensorMap tmB1,
                   const int64_t m_tiles, const int64_t n_tiles, const int64_t k_blocks,
                   const Epi epi, TcStatus* status) {
  static_assert(NA * NB == 2, "one hi/lo split per contraction");
  constexpr uint32_t STAGE_BYTES = NA * A_BYTES + NB * B_BYTES;
  extern __shared__ uint8_t dyn_smem[];
  __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES];
  __shared__ __align__(8) uint64_t tfull_bar[2], tempty_bar[2], drain_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  __shared__ int epi_abort;
  __shared__ __align__(16) uint8_t epi_smem[Epi::kSmemBytes];

  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(dyn_smem) + 1023) &
                                             ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Ctl ctl{&abort_flag, status};

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&full_bar[s]), 1);
      mbar_init(smem_u32(&empty_bar[s]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&tfull_bar[a]), 1);
      mbar_init(smem_u32(&tempty_bar[a]), 128);
    }
    mbar_init(smem_u32(&drain_bar), 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const int64_t num_tiles = m_tiles * n_tiles;

  auto tile_mn = [&](int64_t t, int64_t& m, int64_t& n) {
    if (M_INNER) {
      n = t / m_tiles;
      m = t - n * m_tiles;
    } else {
      m = t / n_tiles;
      n = t - m * n_tiles;
    }
  };

  if (warp == 0) {
    if (lane == 0) {
      // ------------------------------------------------ TMA producer
      int s = 0;
      uint32_t ph = 0;
      int64_t issued = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < num_tiles && ok; t += gridDim.x) {
        int64_t mt, nt;
        tile_mn(t, mt, nt);
        for (int64_t kb = 0; kb < k_blocks; ++kb) {
          if (!bounded_wait(smem_u32(&empty_bar[s]), ph ^ 1, ctl, 1)) {
            ok = false;
            break;
          }
          const uint32_t fb = smem_u32(&full_bar[s]);
          mbar_expect_tx(fb, STAGE_BYTES);
          const uint32_t base = smem_u32(smem + (size_t)s * STAGE_BYTES);
          const int kc = (int)(kb * BK);
          tma_load_2d(base, &tmA0, kc, (int)(mt * BM), fb);
          if (NA == 2) tma_load_2d(base + A_BYTES, &tmA1, kc, (int)(mt * BM), fb);
          const uint32_t bbase = base + NA * A_BYTES;
          tma_load_2d(bbase, &tmB0, kc, (int)(nt * BN), fb);
          if (NB == 2) tma_load_2d(bbase + B_BYTES, &tmB1, kc, (int)(nt * BN), fb);
          ++issued;
          if (++s == STAGES) {
            s = 0;
            ph ^= 1;
          }
        }
      }
      if (!ok) {
        // drain: the last min(issued, STAGES) loads must land before exit
        int64_t n = issued < STAGES ? issued : STAGES;
        int ss = s;
        uint32_t pp = ph;
        for (int64_t i = 0; i < n; ++i) {
          if (--ss < 0) {
            ss = STAGES - 1;
            pp ^= 1;
          }
          const uint64_t t0 = globaltimer();
          while (!mbar_test(smem_u32(&full_bar[ss]), pp) && globaltimer() - t0 < kWaitLimitNs) {
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ------------------------------------------------ MMA issuer
      int s = 0;
      uint32_t ph = 0;
      int64_t i = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < num_tiles && ok; t += gridDim.x, ++i) {
        const int acc = (int)(i & 1);
        const uint32_t aph = (uint32_t)((i >> 1) & 1);
        if (!bounded_wait(smem_u32(&tempty_bar[acc]), aph ^ 1, ctl, 2)) break;
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * BN);
        for (int64_t kb = 0; kb < k_blocks; ++kb) {
          if (!bounded_wait(smem_u32(&full_bar[s]), ph, ctl, 3)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t base = smem_u32(smem + (size_t)s * STAGE_BYTES);
          const uint32_t bbase = base + NA * A_BYTES;
#pragma unroll
          for (int k = 0; k < BK / 16; ++k) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const uint32_t ao = base + (NA == 2 ? q : 0) * A_BYTES + k * 32;
              const uint32_t bo = bbase + (NB == 2 ? q : 0) * B_BYTES + k * 32;
              mma_f16(d, sdesc(ao), sdesc(bo), kIdesc, (kb | k | q) != 0);
            }
          }
          mma_commit(smem_u32(&empty_bar[s]));
          if (++s == STAGES) {
            s = 0;
            ph ^= 1;
          }
        }
        if (ok) mma_commit(smem_u32(&tfull_bar[acc]));
      }
      // every MMA issued by this thread has completed once drain_bar flips
      mma_commit(smem_u32(&drain_bar));
      const uint64_t t0 = globaltimer();
      while (!mbar_test(smem_u32(&drain_bar), 0) && globaltimer() - t0 < kWaitLimitNs) {
      }
    }
  } else {
    // -------------------------------------------------- epilogue warps
    const int quarter = warp & 3;
    const int ep_tid = threadIdx.x - 64;
    Epi e = epi;
    int64_t i = 0;
    for (int64_t t = blockIdx.x; t < num_tiles; t += gridDim.x, ++i) {
      const int acc = (int)(i & 1);
      const uint32_t aph = (uint32_t)((i >> 1) & 1);
      bounded_wait(smem_u32(&tfull_bar[acc]), aph, ctl, 4);
      // the four epilogue warps leave together: a divergent exit would strand
      // the others in the named barriers of tile_begin
      epi_bar();
      if (ep_tid == 0) epi_abort = abort_flag;
      epi_bar();
      if (epi_abort) break;
      tc_fence_after();
      int64_t mt, nt;
      tile_mn(t, mt, nt);
      e.tile_begin(mt, nt, ep_tid, epi_smem);
      e.row_begin(mt * BM + quarter * 32 + lane);
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN);
#pragma unroll 1
      for (int c = 0; c < BN; c += 16) {
        uint32_t v[16];
        tmem_ld16(taddr + c, v);
        tmem_ld_wait();
        e.consume(c, v, epi_smem);
      }
      e.row_end();
      tc_fence_before();
      mbar_arrive(smem_u32(&tempty_bar[acc]));
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// --------------------------------------------------------------- epilogues --

// maximize: row = pattern, column = rotation.  Besides Y it emits, per
// pattern and 256-rotation tile k, the partials of an online log-sum-exp
// relative to the tile maximum m_k:
//   s_k = sum e^(LL-m_k),  d_k = sum e^(LL-m_k) X,  q_k = sum e^(LL-m_k) (LL-m_k)
// with X the scaling denominator term (gaussian: C_rp, poisson: sum W_r).  The
// combine kernel turns them into lse_p, the new scaling and sum P log P.
struct EpiMax {
  static constexpr int kSmemBytes = BN * 8;
  MaxEpiArgs a;
  int64_t n0, ntile, p;
  bool pv;
  float phi, mx, sm, sd, sq;
  double c1, c0;

  __device__ void tile_begin(int64_t mt, int64_t nt, int tid, uint8_t* smem) {
    double* rs = reinterpret_cast<double*>(smem);
    n0 = nt * BN;
    ntile = nt;
    epi_bar();
    for (int c = tid; c < BN; c += 128) {
      const int64_t r = n0 + c;
      rs[c] = r < a.R ? (a.poisson ? a.rowstat[r] : a.rowstat[r] * a.gauss_inv) : 0.0;
    }
    epi_bar();
    (void)mt;
  }
  __device__ void row_begin(int64_t p_) {
    p = p_;
    pv = p < a.N;
    phi = pv ? a.scaling[p] : 1.0f;
    mx = -FLT_MAX;
    sm = sd = sq = 0.0f;
    if (!a.poisson) {
      // LL = (2 C / phi - sum S^2 - sum K^2 / phi^2) / (2 cnt sigma^2)
      c1 = 2.0 * a.gauss_inv / (double)phi;
      c0 = pv ? -a.patstat[p] / ((double)phi * phi) * a.gauss_inv : 0.0;
    }
  }
  __device__ void consume(int c, const uint32_t (&v)[16], uint8_t* smem) {
    const double* rs = reinterpret_cast<const double*>(smem);
    float ll[16], xs[16];
    float cmax = -FLT_MAX;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float x = __uint_as_float(v[k]);
      const int64_t r = n0 + c + k;
      const double l = a.poisson ? (double)x - (double)phi * rs[c + k]
                                 : fma((double)x, c1, c0 - rs[c + k]);
      ll[k] = (float)l;
      xs[k] = a.poisson ? (float)rs[c + k] : x;
      const bool ok = pv && r < a.R;
      if (ok) {
        a.Y[r * a.ldY + p] = a.poisson ? ll[k] : x;
        cmax = fmaxf(cmax, ll[k]);
      } else {
        ll[k] = -FLT_MAX;
      }
    }
    if (cmax > -FLT_MAX) {
      if (cmax > mx) {
        const float f = mx > -FLT_MAX ? expf(mx - cmax) : 0.0f;
        sq = f * (sq + (mx - cmax) * sm);
        sm *= f;
        sd *= f;
        mx = cmax;
      }
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (ll[k] > -FLT_MAX) {
          const float dl = ll[k] - mx;
          const float e = expf(dl);
          sm += e;
          sd = fmaf(e, xs[k], sd);
          sq = fmaf(e, dl, sq);
        }
    }
  }
  __device__ void row_end() {
    if (pv) a.part[ntile * a.N + p] = make_float4(mx, sm, sd, sq);
  }
};

// compress: row = rotation, column = active pixel; inserts into model/weight.
struct EpiCmp {
  static constexpr int kSmemBytes = BN * 16;
  CmpEpiArgs a;
  int64_t j0;
  bool active;
  float m[9];
  float wU, wT;

  __device__ void tile_begin(int64_t mt, int64_t nt, int tid, uint8_t* smem) {
    float4* cs = reinterpret_cast<float4*>(smem);
    j0 = nt * BN;
    epi_bar();
    for (int c = tid; c < BN; c += 128) {
      const int64_t j = j0 + c;
      cs[c] = j < a.npa ? make_float4(a.cx[j], a.cy[j], a.cz[j], a.ins[j] == 1 ? 1.0f : 0.0f)
                        : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    epi_bar();
    (void)mt;
  }
  __device__ void row_begin(int64_t r) {
    active = false;
    if (r < a.R) {
      const float T = a.T[r];
      // emc_atomic.cu:128: rotations with T_r <= 1e-10 are skipped; weight w = rotw T
      if (T > 1e-10f) {
        active = true;
        const float rw = a.rotw[r];
        wT = rw * T;
        wU = wT * a.inv_c0;  // accumulator holds U_r / T_r (rows of P' are divided by T_r)
        emc_voxel::rotation_matrix(a.quat + 4 * r, m);
      }
    }
  }
  __device__ void consume(int c, const uint32_t (&v)[16], uint8_t* smem) {
    if (!active) return;
    const float4* cs = reinterpret_cast<const float4*>(smem);
#pragma unroll 4
    for (int k = 0; k < 16; ++k) {
      const float4 q = cs[c + k];
      if (q.w == 0.0f) continue;
      float u[3];
      emc_voxel::position(m, a.side, q.x, q.y, q.z, u);
      const float val = __uint_as_float(v[k]) * wU;
      if (a.interp == 0) {
        int64_t vox;
        if (!emc_voxel::nearest(u, a.side, 0, &vox)) continue;
        atomicAdd(a.model + vox, val);
        atomicAdd(a.weight + vox, wT);
      } else {
        int64_t vv[8];
        float ww[8];
        const int n = emc_voxel::trilinear(u, a.side, vv, ww);
        for (int cc = 0; cc < n; ++cc) {
          atomicAdd(a.model + vv[cc], ww[cc] * val);
          atomicAdd(a.weight + vv[cc], ww[cc] * wT);
        }
      }
    }
  }
  __device__ void row_end() {}
};

template <int NA, int NB, int STAGES, bool M_INNER, class Epi>
cudaError_t run_gemm(const CUtensorMap& a0, const CUtensorMap& a1, const CUtensorMap& b0,
                     const CUtensorMap& b1, int64_t m_tiles, int64_t n_tiles, int64_t k_blocks,
                     const Epi& epi, TcStatus* st, int num_sms, cudaStream_t stream) {
  constexpr uint32_t stage = NA * A_BYTES + NB * B_BYTES;
  const size_t dyn = (size_t)STAGES * stage + 1024;
  auto kern = tc_gemm_kernel<NA, NB, STAGES, M_INNER, Epi>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  const int64_t tiles = m_tiles * n_tiles;
  if (tiles == 0) return cudaSuccess;
  const int grid = (int)(tiles < num_sms ? tiles : num_sms);
  kern<<<grid, kThreads, dyn, stream>>>(a0, a1, b0, b1, m_tiles, n_tiles, k_blocks, epi, st);
  return cudaGetLastError();
}

// ------------------------------------------------------ responsibility pass --

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Per pattern: lse_p, the new scaling and sum P log P from the tile partials.
//   lse = M + log sum_k s_k e^(m_k - M)
//   D   = sum_k d_k e^(m_k - lse)                       (= sum_r P_rp X_rp)
//   sum_r P log P = sum_k e^(m_k - lse) (q_k + (m_k - lse) s_k)
__global__ void combine_kernel(const RespArgs a) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.N) return;
  float M = -FLT_MAX;
  for (int64_t k = 0; k < a.nparts; ++k) M = fmaxf(M, a.part[k * a.N + p].x);
  double S = 0.0;
  for (int64_t k = 0; k < a.nparts; ++k) {
    const float4 v = a.part[k * a.N + p];
    if (v.y > 0.0f) S += (double)v.y * exp((double)v.x - (double)M);
  }
  const double lse = (double)M + log(S);
  double D = 0.0, Q = 0.0;
  for (int64_t k = 0; k < a.nparts; ++k) {
    const float4 v = a.part[k * a.N + p];
    if (!(v.y > 0.0f)) continue;
    const double dm = (double)v.x - lse;
    const double f = exp(dm);
    D += (double)v.z * f;
    Q += f * ((double)v.w + dm * (double)v.y);
  }
  a.lse[p] = lse;
  a.plogp[p] = Q;
  // emc_cuda.cu:226 for gaussian; poisson MLE sum K / sum_r P_rp sum W_r
  const double num = a.poisson ? a.patsum[p] : a.patstat[p];
  float phi = a.scaling[p];
  if (num > 0.0 && D > 0.0) phi = (float)(num / D);
  a.new_scaling[p] = phi;
}

// LL of one element from the stored Y (poisson: LL itself; gaussian: C).
struct LLFromY {
  int poisson;
  double c1, c0;  // gaussian per-pattern coefficients
  __device__ __forceinline__ double operator()(float y, double rs) const {
    return poisson ? (double)y : fma((double)y, c1, c0 - rs);
  }
};

__device__ __forceinline__ LLFromY make_llf(const RespArgs& a, int64_t p) {
  LLFromY f;
  f.poisson = a.poisson;
  if (!a.poisson && p < a.N) {
    const double phi = a.scaling[p];
    f.c1 = 2.0 * a.gauss_inv / phi;
    f.c0 = -a.patstat[p] / (phi * phi) * a.gauss_inv;
  } else {
    f.c1 = f.c0 = 0.0;
  }
  return f;
}

// One block per rotation r.  Pass 1 reads the row of Y once from HBM, forms
// P_rp = exp(LL_rp - lse_p), keeps it in shared memory and sums T_r.  Pass 2
// writes P'_rp = c0 P_rp / (T_r phi_p) as FP16 hi + lo.  Dividing by T_r (the
// slice average of emc_atomic.cu:105-111) keeps every entry of the row in
// [0, c0/phi_p], so rotations with a tiny total responsibility keep their
// relative precision instead of underflowing FP16.  Rows longer than the
// shared buffer recompute P from Y in pass 2.
constexpr int kRowThreads = 512;
__global__ void __launch_bounds__(kRowThreads) row_kernel(const RespArgs a, int use_smem) {
  extern __shared__ float prow[];
  __shared__ double red[kRowThreads / 32];
  const int64_t r = blockIdx.x;
  const double rs = a.poisson ? a.rowstat[r] : a.rowstat[r] * a.gauss_inv;
  const float* yrow = a.Y + r * a.ldY;
  const int64_t npair = (a.N + 1) / 2;
  auto prob = [&](int64_t p, float y) -> float {
    const LLFromY f = make_llf(a, p);
    return expf((float)(f(y, rs) - a.lse[p]));
  };
  double t = 0.0;
  for (int64_t q = threadIdx.x; q < npair; q += kRowThreads) {
    const int64_t p = 2 * q;
    const float2 y = *reinterpret_cast<const float2*>(yrow + p);
    const float P0 = prob(p, y.x);
    const float P1 = p + 1 < a.N ? prob(p + 1, y.y) : 0.0f;
    if (use_smem) {
      prow[p] = P0;
      prow[p + 1] = P1;
    }
    if (a.P32) {
      a.P32[r * a.N + p] = P0;
      if (p + 1 < a.N) a.P32[r * a.N + p + 1] = P1;
    }
    t += (double)P0 + (double)P1;
  }
  t = warp_sum_d(t);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  double T = 0.0;
  for (int i = 0; i < kRowThreads / 32; ++i) T += red[i];
  if (threadIdx.x == 0) a.T[r] = (float)T;
  const float invT = T > 1e-10 ? (float)(1.0 / T) : 0.0f;
  const int64_t lpair = a.ldP / 2;
  __half2* hi = reinterpret_cast<__half2*>(a.Phi + r * a.ldP);
  __half2* lo = reinterpret_cast<__half2*>(a.Plo + r * a.ldP);
  for (int64_t q = threadIdx.x; q < lpair; q += kRowThreads) {
    const int64_t p = 2 * q;
    float P0 = 0.0f, P1 = 0.0f;
    if (p < a.N) {
      if (use_smem) {
        P0 = prow[p];
        P1 = prow[p + 1];
      } else {
        const float2 y = *reinterpret_cast<const float2*>(yrow + p);
        P0 = prob(p, y.x);
        P1 = p + 1 < a.N ? prob(p + 1, y.y) : 0.0f;
      }
    }
    const float g0 = p < a.N ? a.c0 / a.new_scaling[p] : 0.0f;
    const float g1 = p + 1 < a.N ? a.c0 / a.new_scaling[p + 1] : 0.0f;
    const float x0 = P0 * invT * g0, x1 = P1 * invT * g1;
    const __half h0 = __float2half_rn(x0), h1 = __float2half_rn(x1);
    hi[q] = __halves2half2(h0, h1);
    lo[q] = __halves2half2(__float2half_rn(x0 - __half2float(h0)),
                           __float2half_rn(x1 - __half2float(h1)));
  }
}

__global__ void export_kernel(const RespArgs a, float* P) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.N) return;
  const LLFromY f = make_llf(a, p);
  for (int64_t r = blockIdx.y; r < a.R; r += gridDim.y) {
    const double rs = a.poisson ? a.rowstat[r] : a.rowstat[r] * a.gauss_inv;
    P[r * a.N + p] = (float)exp(f(a.Y[r * a.ldY + p], rs) - a.lse[p]);
  }
}

// Kh[p][j] and Kt[j][p] as FP16 through a 32x32 shared-memory transpose.
__global__ void pack_kernel(const float* K, int64_t N, int64_t npa, int64_t Npad, int64_t Ppad,
                            __half* Kh, __half* Kt, int* bad) {
  __shared__ __half tile[32][33];
  const int64_t j0 = (int64_t)blockIdx.x * 32, p0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  int nbad = 0;
  for (int i = ty; i < 32; i += 8) {
    const int64_t p = p0 + i, j = j0 + tx;
    float k = 0.0f;
    if (p < N && j < npa) {
      k = K[p * npa + j];
      if (!(k >= 0.0f && k <= 2048.0f && k == floorf(k))) nbad++;
    }
    const __half h = __float2half_rn(k);
    tile[i][tx] = h;
    if (p < Npad && j < Ppad) Kh[p * Ppad + j] = h;
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int64_t j = j0 + i, p = p0 + tx;
    if (j < Ppad && p < Npad) Kt[j * Npad + p] = tile[tx][i];
  }
  if (nbad) atomicAdd(bad, nbad);
}

}  // namespace

// ------------------------------------------------------------- host side --

bool tc_encode_2d(CUtensorMap* tm, const void* base, uint64_t inner, uint64_t rows,
                  uint32_t box_rows) {
  typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                               const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                               const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                               CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return false;
    fn = (EncodeFn)p;
  }
  const cuuint64_t dims[2] = {inner, rows};
  const cuuint64_t strides[1] = {inner * 2};
  const cuuint32_t box[2] = {(cuuint32_t)BK, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_maximize_tc(const CUtensorMap& tmK, const CUtensorMap& tmBhi,
                               const CUtensorMap& tmBlo, int64_t Mpad, int64_t Rpad,
                               int64_t Kpad, const MaxEpiArgs& e, TcStatus* status, int num_sms,
                               cudaStream_t st) {
  EpiMax epi;
  epi.a = e;
  // patterns are the inner tile index: the 148 CTAs in flight share B tiles
  return run_gemm<1, 2, 2, true>(tmK, tmK, tmBhi, tmBlo, Mpad / BM, Rpad / BN, Kpad / BK, epi,
                                 status, num_sms, st);
}

cudaError_t launch_compress_tc(const CUtensorMap& tmPhi, const CUtensorMap& tmPlo,
                               const CUtensorMap& tmKt, int64_t Rpad, int64_t Ppad, int64_t Npad,
                               const CmpEpiArgs& e, TcStatus* status, int num_sms,
                               cudaStream_t st) {
  EpiCmp epi;
  epi.a = e;
  // pixel tiles are the inner index: CTAs in flight share the P' tiles
  return run_gemm<2, 1, 3, false>(tmPhi, tmPlo, tmKt, tmKt, Rpad / BM, Ppad / BN, Npad / BK, epi,
                                  status, num_sms, st);
}

cudaError_t launch_resp_pass(RespArgs& a, cudaStream_t st) {
  combine_kernel<<<(unsigned)((a.N + 255) / 256), 256, 0, st>>>(a);
  // the row buffer holds N floats (N rounded up to even) when it fits in shared memory
  const size_t row_bytes = sizeof(float) * (size_t)((a.N + 1) / 2 * 2);
  const int use_smem = row_bytes <= 200 * 1024 ? 1 : 0;
  const size_t dyn = use_smem ? row_bytes : 0;
  cudaError_t e = cudaFuncSetAttribute(row_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(dyn > 0 ? dyn : 1024));
  if (e != cudaSuccess) return e;
  row_kernel<<<(unsigned)a.R, kRowThreads, dyn, st>>>(a, use_smem);
  return cudaGetLastError();
}

cudaError_t launch_resp_export(const RespArgs& a, float* P, cudaStream_t st) {
  dim3 grid((unsigned)((a.N + 255) / 256), (unsigned)(a.R < 4096 ? a.R : 4096));
  export_kernel<<<grid, 256, 0, st>>>(a, P);
  return cudaGetLastError();
}

cudaError_t launch_pack_patterns(const float* K, int64_t N, int64_t npa, int64_t Npad,
                                 int64_t Ppad, __half* Kh, __half* Kt, int* bad, cudaStream_t st) {
  dim3 grid((unsigned)((Ppad + 31) / 32), (unsigned)((Npad + 31) / 32));
  pack_kernel<<<grid, dim3(32, 8), 0, st>>>(K, N, npa, Npad, Ppad, Kh, Kt, bad);
  return cudaGetLastError();
}

}  // namespace emc
