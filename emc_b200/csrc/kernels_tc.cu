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
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <type_traits>

#include "fixed.cuh"
#include "tc.cuh"
#include "voxel.h"

namespace emc {
namespace {

constexpr int BM = 128, BN = 256;
constexpr int kTmemCols = 512;
constexpr uint64_t kWaitLimitNs = 10ull * 1000ull * 1000ull * 1000ull;

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
// Named barrier of the epilogue warps (n threads).
__device__ __forceinline__ void epi_bar(int n = 128) {
  asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory");
}

// Shared-memory matrix descriptor of a K-major operand whose rows are BK FP16
// elements (BK = 64: 128-byte rows, 128B swizzle; BK = 32: 64-byte rows, 64B
// swizzle, as TMA writes them); 8-row core groups 8 * row bytes apart (SBO);
// LBO unused for swizzled K-major layouts; version 1 (sm_100).
template <int BKT>
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  static_assert(BKT == 64 || BKT == 32, "row of 128 or 64 bytes");
  uint64_t d = (uint64_t)((addr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)((8 * BKT * 2) >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)(BKT == 64 ? 2 : 4) << 61;
  return d;
}
// Shared-memory descriptor of an MN-major B operand, 128B swizzle: blocks of
// 64 N-elements (128-byte rows), one row per K index, rows 128 bytes apart so
// 8-row core groups are 1024 bytes apart (SBO), the BN / 64 blocks BKT rows
// of 128 bytes apart (LBO) -- the layout TMA writes for boxes of 64 x BKT.
template <int BKT>
__device__ __forceinline__ uint64_t sdesc_mn(uint32_t addr) {
  uint64_t d = (uint64_t)((addr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((BKT * 128) >> 4) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}
// Instruction descriptor, kind::f16: D = F32, A = B = F16, both K-major.
constexpr uint32_t kIdesc = (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(BN >> 3) << 17) |
                            ((uint32_t)(BM >> 4) << 24);
// The same with B MN-major (bit 16).
constexpr uint32_t kIdescBMN = kIdesc | (1u << 16);

// Epilogues whose B operand is stored MN-major in global memory ([K][N], N
// contiguous) declare kBMajorMN = true.
template <class E, class = void>
struct b_major_mn : std::false_type {};
template <class E>
struct b_major_mn<E, std::void_t<decltype(E::kBMajorMN)>> : std::bool_constant<E::kBMajorMN> {};

// Listed pair epilogues with kCellN = true narrow each tile's MMA to its
// cell's members rounded up to 16 (epi.a.mcnt[cell]); each CTA of the pair
// then holds half of that many B rows.
template <class E, class = void>
struct cell_n : std::false_type {};
template <class E>
struct cell_n<E, std::void_t<decltype(E::kCellN)>> : std::bool_constant<E::kCellN> {};

// Epilogues whose arguments carry gate_count / gate_cap (CmpEpiArgs) return
// from the whole launch unless *gate_count > gate_cap; checked before any
// barrier, TMEM allocation or cluster exchange, so every CTA leaves alike.
template <class E, class = void>
struct has_gate : std::false_type {};
template <class E>
struct has_gate<E, std::void_t<decltype(std::declval<E>().a.gate_count)>> : std::true_type {};
template <class Epi>
__device__ __forceinline__ bool gated_off(const Epi& e) {
  if constexpr (has_gate<Epi>::value)
    return e.a.gate_count && *e.a.gate_count <= (unsigned long long)e.a.gate_cap;
  else
    return false;
}

struct Ctl {
  volatile int* abort;
  TcStatus* st;
};

__device__ bool bounded_wait(uint32_t bar, uint32_t parity, const Ctl& c, int site,
                             uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; ++it) {
    if (mbar_test(bar, parity)) return true;
    if ((it & 31) == 0) {
      if (*c.abort) return false;
      if (globaltimer() - t0 > limit_ns) {
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

// One bounded wait, with a short limit, on an mbarrier that nothing completes:
// the time-out path of bounded_wait (status word, site, early return) that
// every contraction's waits share.  Site 90.
__global__ void wait_probe_kernel(TcStatus* status, uint64_t limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x != 0) return;
  mbar_init(smem_u32(&bar), 1);
  abort_flag = 0;
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  Ctl ctl{&abort_flag, status};
  bounded_wait(smem_u32(&bar), 0, ctl, 90, limit_ns);
}

// ---------------------------------------------------------------- kernel --
template <int NA, int NB, int STAGES, bool M_INNER, int BK, class Epi>
__global__ void __launch_bounds__(64 + 32 * Epi::kEpiWarps, 1)
    tc_gemm_kernel(const __grid_constant__ TmapSet<Epi::kSets> maps,
                   const int64_t m_tiles, const int64_t n_tiles, const int64_t k_blocks,
                   const int raster, const Epi epi, TcStatus* status) {
  static_assert(NA * NB == 2, "one hi/lo split per contraction");
  if (gated_off(epi)) return;
  constexpr bool BMN = b_major_mn<Epi>::value;
  static_assert(!BMN || (NB == 1 && BK == 64 && BN % 64 == 0), "MN-major B: one 64-row operand");
  constexpr uint32_t A_BYTES = BM * BK * 2;
  constexpr uint32_t B_BYTES = BN * BK * 2;
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
      mbar_init(smem_u32(&tempty_bar[a]), 32 * Epi::kEpiWarps);
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

  // Tile order.  The inner index (m for M_INNER, else n) runs fastest, in
  // bands of `raster` outer tiles: the CTAs in flight then cover about
  // gridDim / raster inner tiles x raster outer tiles, so each operand tile
  // they load from HBM is shared through L2 by several of them (the K extent
  // is long, so the panels themselves do not stay in L2).
  auto tile_mn = [&](int64_t t, int64_t& m, int64_t& n) {
    const int64_t inner = M_INNER ? m_tiles : n_tiles;
    const int64_t outer = M_INNER ? n_tiles : m_tiles;
    const int64_t span = (int64_t)raster * inner;
    const int64_t band = t / span;
    const int64_t o0 = band * raster;
    const int64_t g = outer - o0 < raster ? outer - o0 : raster;
    const int64_t w = t - band * span;
    const int64_t o = o0 + w % g, i = w / g;
    if (M_INNER) {
      m = i;
      n = o;
    } else {
      m = o;
      n = i;
    }
  };
  // TMA origins (row and k offset of each operand) and k-block count of tile
  // t: a regular m_tiles x n_tiles grid, or an epilogue-supplied tile list
  // (grouped contractions of uneven groups)
  auto coords = [&](int64_t t, int& ar, int& ak, int& br, int& bk, int64_t& kbs, int& set) {
    if constexpr (Epi::kListed) {
      const TileDesc d = epi.a.tiles[t];
      ar = d.a_row;
      ak = d.a_k0;
      br = d.b_row;
      bk = d.b_k0;
      kbs = d.k_blocks;
      set = d.set;
    } else {
      int64_t mt, nt;
      tile_mn(t, mt, nt);
      ar = (int)(mt * BM);
      ak = 0;
      br = (int)(nt * BN);
      bk = 0;
      kbs = k_blocks;
      set = 0;
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
        int ar, ak, br, bk, set;
        int64_t kbs;
        coords(t, ar, ak, br, bk, kbs, set);
        const CUtensorMap* tA0 = &maps.a0[set];
        const CUtensorMap* tA1 = &maps.a1[set];
        const CUtensorMap* tB0 = &maps.b0[set];
        const CUtensorMap* tB1 = &maps.b1[set];
        for (int64_t kb = 0; kb < kbs; ++kb) {
          if (!bounded_wait(smem_u32(&empty_bar[s]), ph ^ 1, ctl, 1)) {
            ok = false;
            break;
          }
          const uint32_t fb = smem_u32(&full_bar[s]);
          mbar_expect_tx(fb, STAGE_BYTES);
          const uint32_t base = smem_u32(smem + (size_t)s * STAGE_BYTES);
          const int kc = (int)(kb * BK);
          tma_load_2d(base, tA0, ak + kc, ar, fb);
          if (NA == 2) tma_load_2d(base + A_BYTES, tA1, ak + kc, ar, fb);
          const uint32_t bbase = base + NA * A_BYTES;
          if constexpr (BMN) {
            // BN / 64 boxes of 64 N-elements x BK K-rows
#pragma unroll
            for (int i = 0; i < BN / 64; ++i)
              tma_load_2d(bbase + (uint32_t)i * BK * 128, tB0, br + 64 * i, bk + kc, fb);
          } else {
            tma_load_2d(bbase, tB0, bk + kc, br, fb);
            if (NB == 2) tma_load_2d(bbase + B_BYTES, tB1, bk + kc, br, fb);
          }
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
        int ar, ak, br, bk, set;
        int64_t kbs;
        coords(t, ar, ak, br, bk, kbs, set);
        for (int64_t kb = 0; kb < kbs; ++kb) {
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
              if constexpr (BMN) {
                // 16 K-rows of 128 bytes per step
                mma_f16(d, sdesc<BK>(ao), sdesc_mn<BK>(bbase + k * 2048), kIdescBMN,
                        (kb | k | q) != 0);
              } else {
                const uint32_t bo = bbase + (NB == 2 ? q : 0) * B_BYTES + k * 32;
                mma_f16(d, sdesc<BK>(ao), sdesc<BK>(bo), kIdesc, (kb | k | q) != 0);
              }
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
    // TMEM lane quarter = warp % 4; with 8 or 16 epilogue warps, 2 or 4 warps
    // share a quarter and split the columns
    constexpr int EW = Epi::kEpiWarps;
    constexpr int COLS = BN / (EW / 4);
    const int quarter = warp & 3;
    const int ep_tid = threadIdx.x - 64;
    const int col0 = ((warp - 2) / 4) * COLS;
    Epi e = epi;
    int64_t i = 0;
    for (int64_t t = blockIdx.x; t < num_tiles; t += gridDim.x, ++i) {
      const int acc = (int)(i & 1);
      const uint32_t aph = (uint32_t)((i >> 1) & 1);
      bounded_wait(smem_u32(&tfull_bar[acc]), aph, ctl, 4);
      // the epilogue warps leave together: a divergent exit would strand the
      // others in the named barriers of tile_begin
      epi_bar(32 * EW);
      if (ep_tid == 0) epi_abort = abort_flag;
      epi_bar(32 * EW);
      if (epi_abort) break;
      tc_fence_after();
      int64_t mt, nt;
      if constexpr (Epi::kListed) {
        mt = t;  // listed epilogues read their tile descriptor
        nt = 0;
      } else {
        tile_mn(t, mt, nt);
      }
      e.tile_begin(mt, nt, ep_tid, epi_smem);
      e.row_begin(mt * BM + quarter * 32 + lane);
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN);
#pragma unroll 1
      for (int c = col0; c < col0 + COLS; c += 16) {
        uint32_t v[16];
        tmem_ld16(taddr + c, v);
        tmem_ld_wait();
        e.consume(c, v, epi_smem);
      }
      e.row_end();
      tc_fence_before();
      mbar_arrive(smem_u32(&tempty_bar[acc]));
      e.tile_end(mt, nt, ep_tid, epi_smem);
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
// EW = 8 (SM pairs): two warps per TMEM lane quarter, each with half of the
// 256 columns; at the end of a row the second half's running partials are
// merged into the first's through shared memory.
template <int EW>
struct EpiMaxT {
  static constexpr bool kListed = false;
  static constexpr int kSets = 1;
  static constexpr int kEpiWarps = EW;
  static constexpr int kSmemBytes = BN * 8 + (EW == 8 ? BM * 16 : 0);
  MaxEpiArgs a;
  int64_t n0, ntile, p;
  bool pv;
  int half;
  uint8_t* sbuf;
  float phi, mx, sm, sd, sq;
  double c1, c0;

  __device__ void tile_begin(int64_t mt, int64_t nt, int tid, uint8_t* smem) {
    // per column: gaussian sum S^2 * inv (FP64); poisson sum W as an FP32
    // hi + lo pair, so LL = x - phi (hi + lo) takes two FP32 FMAs
    double* rs = reinterpret_cast<double*>(smem);
    float2* rs2 = reinterpret_cast<float2*>(smem);
    n0 = nt * BN;
    ntile = nt;
    half = tid >> 7;
    sbuf = smem;
    epi_bar(32 * EW);
    for (int c = tid; c < BN; c += 32 * EW) {
      const int64_t r = n0 + c;
      const double w = r < a.R ? a.rowstat[r] : 0.0;
      if (a.poisson) {
        const float hi = (float)w;
        rs2[c] = make_float2(hi, (float)(w - (double)hi));
      } else {
        rs[c] = w * a.gauss_inv;
      }
    }
    epi_bar(32 * EW);
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
    const float2* rs2 = reinterpret_cast<const float2*>(smem);
    float ll[16], xs[16];
    float cmax = -FLT_MAX;
    float* yp = a.Y + (n0 + c) * a.ldY + p;
#pragma unroll
    for (int k = 0; k < 16; ++k, yp += a.ldY) {
      const float x = __uint_as_float(v[k]);
      const int64_t r = n0 + c + k;
      if (a.poisson) {
        const float2 w = rs2[c + k];
        ll[k] = fmaf(-phi, w.y, fmaf(-phi, w.x, x));
        xs[k] = w.x + w.y;
      } else {
        ll[k] = (float)fma((double)x, c1, c0 - rs[c + k]);
        xs[k] = x;
      }
      const bool ok = pv && r < a.R;
      if (ok) {
        // a plain store: measured faster than an evict-first (.cs) store here
        *yp = a.poisson ? ll[k] : x;
        cmax = fmaxf(cmax, ll[k]);
      } else {
        ll[k] = -FLT_MAX;
      }
    }
    if (cmax > -FLT_MAX) {
      if (cmax > mx) {
        const float f = mx > -FLT_MAX ? __expf(mx - cmax) : 0.0f;
        sq = f * (sq + (mx - cmax) * sm);
        sm *= f;
        sd *= f;
        mx = cmax;
      }
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (ll[k] > -FLT_MAX) {
          const float dl = ll[k] - mx;
          const float e = __expf(dl);
          sm += e;
          sd = fmaf(e, xs[k], sd);
          sq = fmaf(e, dl, sq);
        }
    }
  }
  __device__ void row_end() {
    if constexpr (EW == 8) {
      // merge the two column halves' partials of this row (log-sum-exp
      // relative to the larger maximum)
      float4* other = reinterpret_cast<float4*>(sbuf + BN * 8);
      const int lr = (int)(p % BM);
      if (half == 1) other[lr] = make_float4(mx, sm, sd, sq);
      epi_bar(32 * EW);
      if (half == 1) return;
      const float4 o = other[lr];
      if (o.x > -FLT_MAX) {
        if (mx > -FLT_MAX) {
          const float m = fmaxf(mx, o.x);
          const float f1 = __expf(mx - m), f2 = __expf(o.x - m);
          sq = f1 * (sq + (mx - m) * sm) + f2 * (o.w + (o.x - m) * o.y);
          sm = f1 * sm + f2 * o.y;
          sd = f1 * sd + f2 * o.z;
          mx = m;
        } else {
          mx = o.x;
          sm = o.y;
          sd = o.z;
          sq = o.w;
        }
      }
    }
    if (pv) a.part[ntile * a.N + p] = make_float4(mx, sm, sd, sq);
  }
  __device__ void tile_end(int64_t, int64_t, int, uint8_t*) {}
};
using EpiMax = EpiMaxT<4>;

// (model, weight) += (x, y) at one voxel as a single vector reduction.
__device__ __forceinline__ void red_add_v2(float2* p, float x, float y) {
  asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(x), "f"(y) : "memory");
}
// The same into the context's accumulators: FP32, or the order-independent
// fixed-point limbs of the deterministic mode.
__device__ __forceinline__ void insert_add(const CmpEpiArgs& e, int64_t vox, float x, float y) {
  if (e.acc64) {
    add_fixed(e.acc64 + 8 * vox, x);
    add_fixed(e.acc64 + 8 * vox + 4, y);
  } else {
    red_add_v2(e.acc + vox, x, y);
  }
}

// compress: row = rotation, column = active pixel; inserts into model/weight.
struct EpiCmp {
  static constexpr bool kListed = false;
  static constexpr int kSets = 1;
  static constexpr int kEpiWarps = 4;
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
      // emc_atomic.cu:128: rotations with T_r <= 1e-10 are skipped (T_r over
      // every pattern shard); weight w = rotw T with this shard's T
      if ((a.Tskip ? a.Tskip[r] : T) > 1e-10f && T > 0.0f) {
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
    // fully unrolled: v[k] stays in registers (a runtime index would put the
    // 16 accumulator words in local memory)
    if (a.interp == 0) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const float4 q = cs[c + k];
        if (q.w == 0.0f) continue;
        float u[3];
        emc_voxel::position(m, a.side, q.x, q.y, q.z, u);
        int64_t vox;
        if (!emc_voxel::nearest(u, a.side, 0, &vox)) continue;
        insert_add(a, vox, __uint_as_float(v[k]) * wU, wT);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const float4 q = cs[c + k];
        if (q.w == 0.0f) continue;
        float u[3];
        emc_voxel::position(m, a.side, q.x, q.y, q.z, u);
        const float val = __uint_as_float(v[k]) * wU;
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          int64_t vox;
          float wc;
          if (!emc_voxel::trilinear_corner(u, a.side, cc, &vox, &wc) || wc == 0.0f) continue;
          insert_add(a, vox, wc * val, wc * wT);
        }
      }
    }
  }
  __device__ void row_end() {}
  __device__ void tile_end(int64_t, int64_t, int, uint8_t*) {}
};

// Grouped maximize of the learned proposal, one tile list over the selected
// cells: row = slot (a (pattern, cell) pair; the cell's slots are contiguous),
// column = member rotation of the cell (<= 256).  Writes Y[slot][member]:
// poisson LL = x - phi_p sum W_r, gaussian cross term x.
struct EpiGMax {
  static constexpr bool kListed = true;
  static constexpr int kSets = 1;
  static constexpr int kEpiWarps = 4;
  static constexpr int kSmemBytes = BN * 8;
  GMaxEpiArgs a;
  TileDesc d;
  int32_t mc, gc;
  int64_t slot;
  bool rv;
  float phi;

  __device__ void tile_begin(int64_t t, int64_t, int tid, uint8_t* smem) {
    float2* rs2 = reinterpret_cast<float2*>(smem);
    d = a.tiles[t];
    mc = a.mcnt[d.cell];
    gc = a.gcnt[d.cell];
    epi_bar();
    for (int c = tid; c < BN; c += 128) {
      const double w = (a.poisson && c < mc) ? a.rowstat[d.b_row + c] : 0.0;
      const float hi = (float)w;
      rs2[c] = make_float2(hi, (float)(w - (double)hi));
    }
    epi_bar();
  }
  __device__ void row_begin(int64_t row) {
    const int local = (int)(row % BM);
    rv = d.local0 + local < gc;
    slot = (int64_t)d.a_row + local;
    phi = rv ? a.scaling[a.gpair[slot]] : 1.0f;
  }
  __device__ void consume(int c, const uint32_t (&v)[16], uint8_t* smem) {
    if (!rv || c >= mc) return;
    const float2* rs2 = reinterpret_cast<const float2*>(smem);
    float y[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const float x = __uint_as_float(v[k]);
      if (a.poisson) {
        const float2 w = rs2[c + k];
        y[k] = fmaf(-phi, w.y, fmaf(-phi, w.x, x));
      } else {
        y[k] = x;
      }
    }
    float* dst = a.Y + slot * a.ldY + c;
    if (c + 16 <= mc) {
#pragma unroll
      for (int k = 0; k < 16; k += 4)
        *reinterpret_cast<float4*>(dst + k) = make_float4(y[k], y[k + 1], y[k + 2], y[k + 3]);
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k)
        if (c + k < mc) dst[k] = y[k];
    }
  }
  __device__ void row_end() {}
  __device__ void tile_end(int64_t, int64_t, int, uint8_t*) {}
};

// The grouped maximize on SM pairs: tiles of 256 slots (a_row, local0 = the
// pair tile's first slot), this CTA's accumulator holds slots 128 rank ..
// 128 rank + 127 of it against all the tile's member columns.
struct EpiGMaxPair : EpiGMax {
  static constexpr bool kCellN = true;  // MMAs as wide as the cell (rounded up to 16)
  __device__ void tile_begin(int64_t t, int64_t x, int tid, uint8_t* smem) {
    EpiGMax::tile_begin(t, x, tid, smem);
    uint32_t rank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    d.a_row += (int32_t)rank * 128;
    d.local0 += (int32_t)rank * 128;
  }
};

// Grouped compress: row = member rotation r of the tile's cell, column =
// active pixel; acc = U_r (the operand rows are P / (T_r phi)), inserted with
// weight rotw T_r as in EpiCmp.
struct EpiGCmp {
  static constexpr bool kListed = true;
  static constexpr int kSets = 1;
  static constexpr bool kBMajorMN = true;  // B = Kg [slot][pixel] read as it lies
  // insertion-heavy epilogue behind short K loops: 16 warps (four per TMEM
  // lane quarter, a quarter of the columns each) keep more reductions in flight
  static constexpr int kEpiWarps = 16;
  static constexpr int kSmemBytes = BN * 16;
  GCmpEpiArgs a;
  TileDesc d;
  int32_t mc;
  bool active;
  float m[9];
  float wT;

  __device__ void tile_begin(int64_t t, int64_t, int tid, uint8_t* smem) {
    float4* cs = reinterpret_cast<float4*>(smem);
    d = a.tiles[t];
    mc = a.mcnt[d.cell];
    epi_bar(32 * kEpiWarps);
    for (int c = tid; c < BN; c += 32 * kEpiWarps) {
      const int64_t j = (int64_t)d.b_row + c;
      cs[c] = j < a.npa ? make_float4(a.cx[j], a.cy[j], a.cz[j], a.ins[j] == 1 ? 1.0f : 0.0f)
                        : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    epi_bar(32 * kEpiWarps);
  }
  __device__ void row_begin(int64_t row) {
    const int local = (int)(row % BM);
    active = false;
    if (d.local0 + local < mc) {
      const int64_t r = (int64_t)d.a_row + local;
      const float T = a.T[r];
      // emc_atomic.cu:128: rotations with T_r <= 1e-10 are skipped; weight w = rotw T
      if (T > 1e-10f) {
        active = true;
        wT = a.rotw[r] * T;
        emc_voxel::rotation_matrix(a.quat + 4 * r, m);
      }
    }
  }
  __device__ void consume(int c, const uint32_t (&v)[16], uint8_t* smem) {
    if (!active) return;
    const float4* cs = reinterpret_cast<const float4*>(smem);
    // fully unrolled: v[k] stays in registers
    if (a.interp == 0) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const float4 q = cs[c + k];
        if (q.w == 0.0f) continue;
        float u[3];
        emc_voxel::position(m, a.side, q.x, q.y, q.z, u);
        int64_t vox;
        if (!emc_voxel::nearest(u, a.side, 0, &vox)) continue;
        red_add_v2(a.acc + vox, __uint_as_float(v[k]) * wT, wT);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const float4 q = cs[c + k];
        if (q.w == 0.0f) continue;
        float u[3];
        emc_voxel::position(m, a.side, q.x, q.y, q.z, u);
        const float val = __uint_as_float(v[k]) * wT;
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          int64_t vox;
          float wc;
          if (!emc_voxel::trilinear_corner(u, a.side, cc, &vox, &wc) || wc == 0.0f) continue;
          red_add_v2(a.acc + vox, wc * val, wc * wT);
        }
      }
    }
  }
  __device__ void row_end() {}
  __device__ void tile_end(int64_t, int64_t, int, uint8_t*) {}
};

inline TmapSet<1> one_set(const CUtensorMap& a0, const CUtensorMap& a1, const CUtensorMap& b0,
                          const CUtensorMap& b1) {
  TmapSet<1> m;
  m.a0[0] = a0;
  m.a1[0] = a1;
  m.b0[0] = b0;
  m.b1[0] = b1;
  return m;
}

// Several datasets in one launch: the tile list's `set` selects the tensor
// maps and the epilogue arguments of its dataset; `local0` is the tile's row
// tile and `cell` its column tile, so the single-dataset epilogues run as
// they are.
struct EpiBatchMax {
  static constexpr bool kListed = true;
  static constexpr int kSets = kMaxBatch;
  static constexpr int kEpiWarps = 4;
  static constexpr int kSmemBytes = EpiMax::kSmemBytes;
  BatchMaxArgs a;
  EpiMax inner;
  int64_t row0;

  __device__ void tile_begin(int64_t t, int64_t, int tid, uint8_t* smem) {
    const TileDesc d = a.tiles[t];
    inner.a = a.set[d.set];
    row0 = (int64_t)d.local0 * BM;
    inner.tile_begin(d.local0, d.cell, tid, smem);
  }
  __device__ void row_begin(int64_t row) { inner.row_begin(row0 + row % BM); }
  __device__ void consume(int c, const uint32_t (&v)[16], uint8_t* smem) { inner.consume(c, v, smem); }
  __device__ void row_end() { inner.row_end(); }
  __device__ void tile_end(int64_t, int64_t, int, uint8_t*) {}
};

struct EpiBatchCmp {
  static constexpr bool kListed = true;
  static constexpr int kSets = kMaxBatch;
  static constexpr int kEpiWarps = 4;
  static constexpr int kSmemBytes = EpiCmp::kSmemBytes;
  BatchCmpArgs a;
  EpiCmp inner;
  int64_t row0;

  __device__ void tile_begin(int64_t t, int64_t, int tid, uint8_t* smem) {
    const TileDesc d = a.tiles[t];
    inner.a = a.set[d.set];
    row0 = (int64_t)d.local0 * BM;
    inner.tile_begin(d.local0, d.cell, tid, smem);
  }
  __device__ void row_begin(int64_t row) { inner.row_begin(row0 + row % BM); }
  __device__ void consume(int c, const uint32_t (&v)[16], uint8_t* smem) { inner.consume(c, v, smem); }
  __device__ void row_end() { inner.row_end(); }
  __device__ void tile_end(int64_t, int64_t, int, uint8_t*) {}
};

// The batched maximize on SM pairs: the tile's local0 is its 256-row pair
// tile, so this CTA's 128-row block is 2 local0 + rank.
struct EpiBatchMaxPair {
  static constexpr bool kListed = true;
  static constexpr int kSets = kMaxBatch;
  static constexpr int kEpiWarps = 4;
  static constexpr int kSmemBytes = EpiMax::kSmemBytes;
  BatchMaxArgs a;
  EpiMax inner;
  int64_t row0;

  __device__ void tile_begin(int64_t t, int64_t, int tid, uint8_t* smem) {
    const TileDesc d = a.tiles[t];
    inner.a = a.set[d.set];
    uint32_t rank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    const int64_t mrow = (int64_t)d.local0 * 2 + rank;
    row0 = mrow * BM;
    inner.tile_begin(mrow, d.cell, tid, smem);
  }
  __device__ void row_begin(int64_t row) { inner.row_begin(row0 + row); }
  __device__ void consume(int c, const uint32_t (&v)[16], uint8_t* smem) { inner.consume(c, v, smem); }
  __device__ void row_end() { inner.row_end(); }
  __device__ void tile_end(int64_t, int64_t, int, uint8_t*) {}
};

// The batched compress on SM pairs (256-rotation pair tiles).
struct EpiBatchCmpPair {
  static constexpr bool kListed = true;
  static constexpr int kSets = kMaxBatch;
  static constexpr int kEpiWarps = 4;
  static constexpr int kSmemBytes = EpiCmp::kSmemBytes;
  BatchCmpArgs a;
  EpiCmp inner;
  int64_t row0;

  __device__ void tile_begin(int64_t t, int64_t, int tid, uint8_t* smem) {
    const TileDesc d = a.tiles[t];
    inner.a = a.set[d.set];
    uint32_t rank;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(rank));
    const int64_t mrow = (int64_t)d.local0 * 2 + rank;
    row0 = mrow * BM;
    inner.tile_begin(mrow, d.cell, tid, smem);
  }
  __device__ void row_begin(int64_t row) { inner.row_begin(row0 + row); }
  __device__ void consume(int c, const uint32_t (&v)[16], uint8_t* smem) { inner.consume(c, v, smem); }
  __device__ void row_end() { inner.row_end(); }
  __device__ void tile_end(int64_t, int64_t, int, uint8_t*) {}
};

template <int NA, int NB, int STAGES, bool M_INNER, int BK, class Epi>
cudaError_t run_gemm(const TmapSet<Epi::kSets>& maps, int64_t m_tiles, int64_t n_tiles,
                     int64_t k_blocks, const Epi& epi, TcStatus* st, int num_sms,
                     cudaStream_t stream, int raster = 1) {
  if (raster < 1) raster = 1;
  constexpr uint32_t stage = NA * BM * BK * 2 + NB * BN * BK * 2;
  const size_t dyn = (size_t)STAGES * stage + 1024;
  auto kern = tc_gemm_kernel<NA, NB, STAGES, M_INNER, BK, Epi>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  const int64_t tiles = m_tiles * n_tiles;
  if (tiles == 0) return cudaSuccess;
  const int grid = (int)(tiles < num_sms ? tiles : num_sms);
  kern<<<grid, 64 + 32 * Epi::kEpiWarps, dyn, stream>>>(maps, m_tiles, n_tiles, k_blocks, raster,
                                                       epi, st);
  return cudaGetLastError();
}

// ---------------------------------------------- two-SM maximize contraction --
// The maximize contraction on SM pairs (cta_group::2, cluster of 2): a pair
// computes a 256-pattern x 256-rotation tile with one tcgen05.mma per 16-wide
// K step and operand half; each CTA loads its 128 patterns of the counts and
// its 128 rotations of the hi and lo slice operand, so every SM moves half
// the slice bytes of the one-SM kernel through shared memory, which leaves
// room for 128-byte K-steps (4 stages of 48 KB).  The leader (rank 0) issues
// the MMAs; both CTAs' TMA loads complete on the leader's barriers; the
// leader's commits release both CTAs' stages and accumulators; each CTA's
// epilogue drains its own 128 TMEM lanes (its patterns) x 256 rotations.

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// Address of the same shared-memory object in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t peer_addr(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// TMA load into this CTA's shared memory completing on the pair leader's barrier.
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* tm, int c0, int c1,
                                                 uint32_t bar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)tm), "r"(c0), "r"(c1), "r"(bar_cluster)
      : "memory");
}
__device__ __forceinline__ void mma_f16_pair(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                             uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}
// Arrive on an mbarrier (this CTA's or the peer's, shared::cluster address)
// once every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit_pair(uint32_t bar_cluster) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar_cluster)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster)
               : "memory");
}

// M = 256 (the pair), N = 256.
constexpr uint32_t kIdescPair = (1u << 4) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(256 >> 4) << 24);
constexpr int kPairBK = 64;
constexpr int kPairStages = 4;

// NA / NB: 1, or 2 for an operand split into FP16 hi + lo (one of them).
// A listed epilogue (Epi::kListed) supplies the tiles: TileDesc rows of the
// pair (a_row, b_row: the CTA adds 128 x rank), k-block count and tensor-map
// set; its row_begin then receives the row inside this CTA's 128 rows.
template <int NA, int NB, bool M_INNER, class Epi>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(64 + 32 * Epi::kEpiWarps, 1)
    tc_pair_kernel(const __grid_constant__ TmapSet<Epi::kSets> maps, const int64_t m_tiles,
                   const int64_t n_tiles, const int64_t k_blocks, const int raster,
                   const Epi epi, TcStatus* status) {
  static_assert(NA * NB == 2, "one hi/lo split per contraction");
  if (gated_off(epi)) return;
  constexpr uint32_t A_BYTES = 128 * kPairBK * 2;   // this CTA's 128 rows of A
  constexpr uint32_t B_BYTES = 128 * kPairBK * 2;   // this CTA's 128 rows (half) of B
  constexpr uint32_t STAGE_BYTES = NA * A_BYTES + NB * B_BYTES;
  constexpr int STAGES = kPairStages;
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
  const uint32_t rank = cluster_rank();
  const bool leader = rank == 0;
  Ctl ctl{&abort_flag, status};
  // stop the peer too: its waits then end at their next check
  auto abort_pair = [&]() {
    abort_flag = 1;
    const uint32_t pa = peer_addr(smem_u32(&abort_flag), rank ^ 1u);
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(pa), "r"(1) : "memory");
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&full_bar[s]), 1);
      mbar_init(smem_u32(&empty_bar[s]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&tfull_bar[a]), 1);
      mbar_init(smem_u32(&tempty_bar[a]), 2);  // one arrival per CTA's epilogue
    }
    mbar_init(smem_u32(&drain_bar), 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // both CTAs' barriers exist before any remote arrival or load
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const int64_t num_tiles = m_tiles * n_tiles;
  const int64_t cid = blockIdx.x >> 1, ncl = gridDim.x >> 1;

  // the inner index (m for M_INNER, else n) fastest, in bands of `raster`
  // outer tiles (as tile_mn of tc_gemm_kernel)
  auto tile_mn = [&](int64_t t, int64_t& m, int64_t& n) {
    const int64_t inner = M_INNER ? m_tiles : n_tiles;
    const int64_t outer = M_INNER ? n_tiles : m_tiles;
    const int64_t span = (int64_t)raster * inner;
    const int64_t band = t / span;
    const int64_t o0 = band * raster;
    const int64_t g = outer - o0 < raster ? outer - o0 : raster;
    const int64_t w = t - band * span;
    const int64_t o = o0 + w % g, i = w / g;
    if (M_INNER) {
      m = i;
      n = o;
    } else {
      m = o;
      n = i;
    }
  };

  if (warp == 0) {
    if (lane == 0) {
      // ------------------------------------------------ TMA producer (both CTAs)
      int s = 0;
      uint32_t ph = 0;
      int64_t issued = 0;
      bool ok = true;
      for (int64_t t = cid; t < num_tiles && ok; t += ncl) {
        int ar, br, set = 0;
        int64_t kbs = k_blocks;
        if constexpr (Epi::kListed) {
          const TileDesc d = epi.a.tiles[t];
          ar = d.a_row + (int)rank * 128;
          br = d.b_row + (int)rank * 128;
          if constexpr (cell_n<Epi>::value)
            br = d.b_row + (int)rank * (((epi.a.mcnt[d.cell] + 15) & ~15) / 2);
          kbs = d.k_blocks;
          set = d.set;
        } else {
          int64_t mt, nt;
          tile_mn(t, mt, nt);
          ar = (int)(mt * 256 + rank * 128);
          br = (int)(nt * 256 + rank * 128);
        }
        const CUtensorMap* tA0 = &maps.a0[set];
        const CUtensorMap* tA1 = &maps.a1[set];
        const CUtensorMap* tB0 = &maps.b0[set];
        const CUtensorMap* tB1 = &maps.b1[set];
        for (int64_t kb = 0; kb < kbs; ++kb) {
          if (!bounded_wait(smem_u32(&empty_bar[s]), ph ^ 1, ctl, 1)) {
            ok = false;
            break;
          }
          const uint32_t fb = smem_u32(&full_bar[s]);
          if (leader) mbar_expect_tx(fb, 2 * STAGE_BYTES);  // both CTAs' bytes
          const uint32_t fb_leader = peer_addr(fb, 0);
          const uint32_t base = smem_u32(smem + (size_t)s * STAGE_BYTES);
          const int kc = (int)(kb * kPairBK);
          tma_load_2d_pair(base, tA0, kc, ar, fb_leader);
          if (NA == 2) tma_load_2d_pair(base + A_BYTES, tA1, kc, ar, fb_leader);
          const uint32_t bbase = base + NA * A_BYTES;
          tma_load_2d_pair(bbase, tB0, kc, br, fb_leader);
          if (NB == 2) tma_load_2d_pair(bbase + B_BYTES, tB1, kc, br, fb_leader);
          ++issued;
          if (++s == STAGES) {
            s = 0;
            ph ^= 1;
          }
        }
      }
      if (!ok) {
        abort_pair();
        if (leader) {
          // the last min(issued, STAGES) stages must land (both CTAs' bytes
          // complete on these barriers) before the pair exits
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
        } else {
          // the peer cannot observe its loads; give them time to land
          const uint64_t t0 = globaltimer();
          while (globaltimer() - t0 < 2000000ull) {
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && leader) {
      // ------------------------------------------------ MMA issuer (leader)
      int s = 0;
      uint32_t ph = 0;
      int64_t i = 0;
      bool ok = true;
      for (int64_t t = cid; t < num_tiles && ok; t += ncl, ++i) {
        const int acc = (int)(i & 1);
        const uint32_t aph = (uint32_t)((i >> 1) & 1);
        if (!bounded_wait(smem_u32(&tempty_bar[acc]), aph ^ 1, ctl, 2)) {
          abort_pair();
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * BN);
        int64_t kbs = k_blocks;
        uint32_t idesc = kIdescPair;
        if constexpr (Epi::kListed) {
          const TileDesc td = epi.a.tiles[t];
          kbs = td.k_blocks;
          if constexpr (cell_n<Epi>::value) {
            // N = the cell's members rounded up to 16 (bits 17..22: N >> 3)
            const uint32_t n16 = (uint32_t)((epi.a.mcnt[td.cell] + 15) & ~15);
            idesc = (kIdescPair & ~(0x3Fu << 17)) | ((n16 >> 3) << 17);
          }
        }
        for (int64_t kb = 0; kb < kbs; ++kb) {
          if (!bounded_wait(smem_u32(&full_bar[s]), ph, ctl, 3)) {
            ok = false;
            abort_pair();
            break;
          }
          tc_fence_after();
          const uint32_t base = smem_u32(smem + (size_t)s * STAGE_BYTES);
          const uint32_t bbase = base + NA * A_BYTES;
#pragma unroll
          for (int k = 0; k < kPairBK / 16; ++k) {
#pragma unroll
            for (int q = 0; q < 2; ++q)
              mma_f16_pair(d, sdesc<kPairBK>(base + (NA == 2 ? q : 0) * A_BYTES + k * 32),
                           sdesc<kPairBK>(bbase + (NB == 2 ? q : 0) * B_BYTES + k * 32),
                           idesc, (kb | k | q) != 0);
          }
          // release this stage in both CTAs once its MMAs are done
          const uint32_t eb = smem_u32(&empty_bar[s]);
          mma_commit_pair(peer_addr(eb, 0));
          mma_commit_pair(peer_addr(eb, 1));
          if (++s == STAGES) {
            s = 0;
            ph ^= 1;
          }
        }
        if (ok) {
          const uint32_t tb = smem_u32(&tfull_bar[acc]);
          mma_commit_pair(peer_addr(tb, 0));
          mma_commit_pair(peer_addr(tb, 1));
        }
      }
      mma_commit_pair(peer_addr(smem_u32(&drain_bar), 0));
      const uint64_t t0 = globaltimer();
      while (!mbar_test(smem_u32(&drain_bar), 0) && globaltimer() - t0 < kWaitLimitNs) {
      }
    }
  } else {
    // -------------------------------------------------- epilogue warps (both CTAs)
    // TMEM lane quarter = warp % 4; with 8 epilogue warps two share a quarter
    // and take one half of the columns each
    constexpr int EW = Epi::kEpiWarps;
    static_assert(EW == 4 || EW == 8, "4 or 8 epilogue warps");
    constexpr int COLS = BN / (EW / 4);
    const int quarter = warp & 3;
    const int ep_tid = threadIdx.x - 64;
    const int col0 = ((warp - 2) / 4) * COLS;
    Epi e = epi;
    int64_t i = 0;
    const uint32_t tempty_leader0 = peer_addr(smem_u32(&tempty_bar[0]), 0);
    const uint32_t tempty_leader1 = peer_addr(smem_u32(&tempty_bar[1]), 0);
    for (int64_t t = cid; t < num_tiles; t += ncl, ++i) {
      const int acc = (int)(i & 1);
      const uint32_t aph = (uint32_t)((i >> 1) & 1);
      bounded_wait(smem_u32(&tfull_bar[acc]), aph, ctl, 4);
      epi_bar(32 * EW);
      if (ep_tid == 0) epi_abort = abort_flag;
      epi_bar(32 * EW);
      if (epi_abort) break;
      tc_fence_after();
      int64_t mt = t, nt = 0;
      if constexpr (Epi::kListed) {
        e.tile_begin(t, 0, ep_tid, epi_smem);
        e.row_begin(quarter * 32 + lane);
      } else {
        tile_mn(t, mt, nt);
        const int64_t mrow = mt * 2 + rank;  // this CTA's 128-row block
        e.tile_begin(mrow, nt, ep_tid, epi_smem);
        e.row_begin(mrow * BM + quarter * 32 + lane);
      }
      const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN);
#pragma unroll 1
      for (int c = col0; c < col0 + COLS; c += 16) {
        uint32_t v[16];
        tmem_ld16(taddr + c, v);
        tmem_ld_wait();
        e.consume(c, v, epi_smem);
      }
      e.row_end();
      tc_fence_before();
      epi_bar(32 * EW);  // the whole accumulator of this CTA has been read
      if (ep_tid == 0) mbar_arrive_cluster(acc ? tempty_leader1 : tempty_leader0);
      e.tile_end(mt, nt, ep_tid, epi_smem);
    }
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync();  // neither CTA leaves while the pair's MMAs or loads may touch it
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

template <int NA, int NB, bool M_INNER, class Epi>
cudaError_t run_pair(const TmapSet<Epi::kSets>& maps, int64_t m_tiles, int64_t n_tiles,
                     int64_t k_blocks, const Epi& epi, TcStatus* st, int num_sms,
                     cudaStream_t stream, int raster) {
  constexpr uint32_t stage = 128 * kPairBK * 2 * (NA + NB);
  const size_t dyn = (size_t)kPairStages * stage + 1024;
  auto kern = tc_pair_kernel<NA, NB, M_INNER, Epi>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  if (e != cudaSuccess) return e;
  const int64_t tiles = m_tiles * n_tiles;
  if (tiles == 0) return cudaSuccess;
  const int64_t pairs = num_sms / 2;
  const int grid = 2 * (int)(tiles < pairs ? tiles : pairs);
  kern<<<grid, 64 + 32 * Epi::kEpiWarps, dyn, stream>>>(maps, m_tiles, n_tiles, k_blocks,
                                        raster < 1 ? 1 : raster, epi, st);
  return cudaGetLastError();
}

// ------------------------------------------------------ responsibility pass --

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

// The two sweeps over Y are tiled 32 rotations x 1024 patterns per block:
// each thread owns four consecutive patterns (one float4 of Y per row), loads
// their constants (lse, LL coefficients, 1/phi) once and reuses them for the
// block's 32 rows.
constexpr int kSweepRows = 32;
constexpr int kSweepThreads = 256;
constexpr int kSweepPatterns = 4 * kSweepThreads;

// Per-pattern constants of the sweeps.  Poisson Y is the LL itself, so only
// lse is kept (fewer registers, more warps in flight); gaussian keeps the
// coefficients of LL = (2 C / phi - sum S^2 - sum K^2 / phi^2) * inv.
template <bool POISSON>
struct PatConst {
  double lse[4];
  float lse_hi[4], lse_lo[4];  // poisson: lse = hi + lo, hi = lse rounded to FP32
  double c1[4], c0[4];  // gaussian only
  bool ok[4];
};

template <bool POISSON>
__device__ __forceinline__ void load_consts(const RespArgs& a, int64_t p0, PatConst<POISSON>& k) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t p = p0 + i;
    k.ok[i] = p < a.N;
    k.lse[i] = k.ok[i] ? a.lse[p] : 0.0;
    k.lse_hi[i] = (float)k.lse[i];
    k.lse_lo[i] = (float)(k.lse[i] - (double)k.lse_hi[i]);
    if constexpr (!POISSON) {
      const LLFromY f = make_llf(a, p);
      k.c1[i] = f.c1;
      k.c0[i] = f.c0;
    }
  }
}

// P = exp(LL - lse), exp in FP32.  LL and lse are ~1e4, so the difference
// needs more than FP32: gaussian, in FP64; poisson (LL = y, an FP32 value),
// as (y - hi) - lo with lse = hi + lo split into FP32 parts: y - hi is exact
// whenever y lies within a factor of two of hi (Sterbenz), which holds for
// every entry that does not underflow, and the one rounding left is the
// one the FP64 difference gets when it is rounded to FP32.
template <bool POISSON>
__device__ __forceinline__ void probs_from(const PatConst<POISSON>& k, float4 y, double rs,
                                           float (&P)[4]) {
  const float yy[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float d;
    if constexpr (POISSON)
      d = __fsub_rn(__fsub_rn(yy[i], k.lse_hi[i]), k.lse_lo[i]);
    else
      d = (float)(fma((double)yy[i], k.c1[i], k.c0[i] - rs) - k.lse[i]);
    P[i] = k.ok[i] ? expf(d) : 0.0f;
  }
}

// Sweep A: Tpart[pattern block][r] = sum over the block's patterns of P_rp.
template <bool POISSON>
__global__ void __launch_bounds__(kSweepThreads, 4) rowsum_kernel(const RespArgs a) {
  __shared__ float red[kSweepThreads / 32][kSweepRows];
  // Each warp gathers the compacted entries of its rows in shared memory and
  // reserves room for them with one atomic per flush: one counter serves the
  // whole grid, and an atomic per warp and row on it serialised the sweep
  // (measured at full size: 15.0 -> 10.6 ms per steady-state iteration)
  constexpr int kBuf = 256;
  __shared__ int2 brp[kSweepThreads / 32][kBuf];
  __shared__ float bv[kSweepThreads / 32][kBuf];
  const int64_t p0 = (int64_t)blockIdx.x * kSweepPatterns + 4 * threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.y * kSweepRows;
  const bool any = p0 < a.N;
  PatConst<POISSON> k;
  load_consts<POISSON>(a, p0, k);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int nb = 0;  // entries in this warp's buffer (warp-uniform)
  auto flush = [&]() {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(a.list_count, (unsigned long long)nb);
    base = __shfl_sync(0xffffffffu, base, 0);
    __syncwarp();
    for (int e = lane; e < nb; e += 32) {
      const int64_t pos = (int64_t)base + e;
      if (pos < a.list_cap) {
        a.list_rp[pos] = brp[w][e];
        a.list_P[pos] = bv[w][e];
      }
    }
    __syncwarp();
    nb = 0;
  };
  // four rows per step: their loads are issued before any result is needed
  for (int i0 = 0; i0 < kSweepRows; i0 += 4) {
    float t[4];
    float4 y[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t r = r0 + i0 + u;
      y[u] = (r < a.R && any) ? *reinterpret_cast<const float4*>(a.Y + r * a.ldY + p0)
                              : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t r = r0 + i0 + u;
      t[u] = 0.0f;
      float P[4] = {0.f, 0.f, 0.f, 0.f};
      if (r < a.R && any) {
        const double rs = POISSON ? 0.0 : a.rowstat[r] * a.gauss_inv;
        probs_from<POISSON>(k, y[u], rs, P);
        t[u] = (P[0] + P[1]) + (P[2] + P[3]);
      }
      if (a.list_count) {
        int n = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) n += (k.ok[j] && P[j] >= a.list_min) ? 1 : 0;
        if (__any_sync(0xffffffffu, n > 0)) {
          int inc = n;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
          }
          const int tot = __shfl_sync(0xffffffffu, inc, 31);
          if (nb + tot > kBuf) flush();
          int q = nb + inc - n;
          const float yy[4] = {y[u].x, y[u].y, y[u].z, y[u].w};
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (k.ok[j] && P[j] >= a.list_min) {
              brp[w][q] = make_int2((int)(a.list_r0 + r), (int)(p0 + j));
              bv[w][q] = a.list_store_y ? yy[j] : P[j];
              ++q;
            }
          nb += tot;
          __syncwarp();
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t[u] += __shfl_xor_sync(0xffffffffu, t[u], o);
      if (lane == 0) red[w][i0 + u] = t[u];
    }
  }
  if (a.list_count && nb > 0) flush();
  __syncthreads();
  if (threadIdx.x < kSweepRows) {
    const int64_t r = r0 + threadIdx.x;
    float t = 0.0f;
    for (int i = 0; i < kSweepThreads / 32; ++i) t += red[i][threadIdx.x];
    if (r < a.R && a.Tpart) a.Tpart[(int64_t)blockIdx.x * a.R + r] = t;
  }
}

// Sweep B: P'_rp = c0 P_rp / (T_r phi_p) as FP16 hi + lo.  Dividing each row
// by its total responsibility T_r (the slice average of emc_atomic.cu:105-111)
// keeps every entry in [0, c0/phi_p], so rotations with a tiny T_r keep their
// relative precision instead of underflowing FP16.
template <bool POISSON>
__device__ __forceinline__ void write_tile(const RespArgs& a, int64_t nblk, int64_t bx,
                                           int64_t by, float* invT) {
  const int64_t p0 = bx * kSweepPatterns + 4 * threadIdx.x;
  const int64_t r0 = by * kSweepRows;
  __syncthreads();  // the previous tile's invT is read
  if (threadIdx.x < kSweepRows) {
    const int64_t r = r0 + threadIdx.x;
    double T = 0.0;
    if (r < a.R) {
      for (int64_t b = 0; b < nblk; ++b) T += a.Tpart[b * a.R + r];
      if (bx == 0) a.T[r] = (float)T;
    }
    // P <= T, so P / T stays finite; the insertion decides which rows count
    invT[threadIdx.x] = T > 1e-30 ? (float)(1.0 / T) : 0.0f;
  }
  __syncthreads();
  if (p0 >= a.ldP) return;
  PatConst<POISSON> k;
  load_consts<POISSON>(a, p0, k);
  float g[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) g[i] = k.ok[i] ? a.c0 / a.new_scaling[p0 + i] : 0.0f;
  const bool any = p0 < a.N;
  for (int i0 = 0; i0 < kSweepRows; i0 += 4) {
    float4 y[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t r = r0 + i0 + u;
      y[u] = (r < a.R && any) ? *reinterpret_cast<const float4*>(a.Y + r * a.ldY + p0)
                              : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
    const int i = i0 + u;
    const int64_t r = r0 + i;
    if (r >= a.R) break;
    float P[4] = {0.f, 0.f, 0.f, 0.f};
    if (any) {
      const double rs = POISSON ? 0.0 : a.rowstat[r] * a.gauss_inv;
      probs_from<POISSON>(k, y[u], rs, P);
    }
    __half h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float x = P[j] * invT[i] * g[j];
      h[j] = __float2half_rn(x);
      l[j] = __float2half_rn(x - __half2float(h[j]));
    }
    uint2 hv, lv;
    hv.x = (uint32_t)__half_as_ushort(h[0]) | ((uint32_t)__half_as_ushort(h[1]) << 16);
    hv.y = (uint32_t)__half_as_ushort(h[2]) | ((uint32_t)__half_as_ushort(h[3]) << 16);
    lv.x = (uint32_t)__half_as_ushort(l[0]) | ((uint32_t)__half_as_ushort(l[1]) << 16);
    lv.y = (uint32_t)__half_as_ushort(l[2]) | ((uint32_t)__half_as_ushort(l[3]) << 16);
    __stcs(reinterpret_cast<uint2*>(a.Phi + r * a.ldP + p0), hv);
    __stcs(reinterpret_cast<uint2*>(a.Plo + r * a.ldP + p0), lv);
    if (a.P32) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (k.ok[j]) a.P32[r * a.N + p0 + j] = P[j];
    }
    }
  }
}

// Tiles of kSweepPatterns columns x kSweepRows rows, tile t = (t % wblk, t /
// wblk); a block takes tiles blockIdx.x, + gridDim.x, ...  Launched one tile
// per block, or, gated, on a small grid (a launch whose gate stays closed
// then costs a few thousand empty blocks, not one per tile).
template <bool POISSON>
__global__ void __launch_bounds__(kSweepThreads, 4) write_kernel(const RespArgs a, int64_t nblk,
                                                                 int64_t wblk, int64_t ntiles) {
  if (a.gate_count && *a.gate_count <= (unsigned long long)a.gate_cap) return;
  __shared__ float invT[kSweepRows];
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t bx = t % wblk, by = t / wblk;
    write_tile<POISSON>(a, nblk, bx, by, invT);
  }
}

// ------------------------------------------------ responsibility lists --
// The compress operand as lists: for every rotation r the patterns p with
// P_rp >= list_min and x_rp = P_rp / (T_r phi_p) (the value write_kernel
// stores in P').  Posteriors are sharp, so there are a few per pattern
// against R per pattern in P'.  rowsum_kernel compacts the entries while it
// sums the rows; a counting sort orders them by rotation.

// rowoff[0..R] = exclusive prefix sums of rowtot; one block of 1024 threads,
// each with a contiguous run of rows.
__global__ void __launch_bounds__(1024) list_rowscan_kernel(const int64_t* rowtot, int64_t R,
                                                            int64_t* rowoff) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t chunk = (R + 1023) / 1024, beg = t * chunk, end = beg + chunk < R ? beg + chunk : R;
  int64_t s = 0;
  for (int64_t r = beg; r < end; ++r) s += rowtot[r];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int64_t v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int64_t run = part[t] - s;
  for (int64_t r = beg; r < end; ++r) {
    rowoff[r] = run;
    run += rowtot[r];
  }
  if (t == 1023) rowoff[R] = part[1023];
}

// Exclusive prefix sums of long arrays in three launches: per block of
// kScanBlock elements its total, one block scanning the totals
// (list_rowscan_kernel), then each block's elements from its offset.
constexpr int kScanPer = 8;
constexpr int kScanBlock = 1024 * kScanPer;

__global__ void __launch_bounds__(1024) scan_totals_kernel(const int64_t* in, int64_t n,
                                                           int64_t* tot) {
  __shared__ int64_t red[32];
  const int64_t b0 = (int64_t)blockIdx.x * kScanBlock + (int64_t)threadIdx.x * kScanPer;
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k)
    if (b0 + k < n) s += in[b0 + k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int64_t v = red[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) tot[blockIdx.x] = v;
  }
}

__global__ void __launch_bounds__(1024) scan_apply_kernel(const int64_t* in, int64_t n,
                                                          const int64_t* boff, int64_t* out) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t b0 = (int64_t)blockIdx.x * kScanBlock + (int64_t)t * kScanPer;
  int64_t v[kScanPer], s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    v[k] = b0 + k < n ? in[b0 + k] : 0;
    s += v[k];
  }
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int64_t x = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += x;
    __syncthreads();
  }
  int64_t run = boff[blockIdx.x] + part[t] - s;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (b0 + k < n) out[b0 + k] = run;
    run += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && t == 0) out[n] = boff[gridDim.x];  // the total
}

// T_r from the row-sum partials (FP64 sum in pattern-block order, as
// write_kernel forms it).
__global__ void finish_T_kernel(const float* Tpart, int64_t nblk, int64_t R, float* T) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  double t = 0.0;
  for (int64_t b = 0; b < nblk; ++b) t += Tpart[b * R + r];
  T[r] = (float)t;
}

// Counting sort of the compacted entries by rotation: STEP 0 counts per
// rotation, STEP 1 writes (pattern, x) at rowoff[r] + cursor.
// Entries below rel_min T_r are dropped: each moves its rotation's slice sum
// by less than rel_min.
template <int STEP>
__global__ void compact_sort_kernel(const int2* rp, const float* Pv, int64_t n, const float* T,
                                    const float* new_scaling, float rel_min,
                                    unsigned long long* cnt, const int64_t* rowoff, int32_t* pat,
                                    float* xv, const unsigned long long* n_dev) {
  if (n_dev) {  // the count on the device; above the capacity n the lists stay empty
    const unsigned long long c = *n_dev;
    if (c > (unsigned long long)n) return;
    n = (int64_t)c;
  }
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int2 v = rp[e];
    const float Tr = T[v.x], P = Pv[e];
    if (!(Tr > 0.0f) || !(P >= rel_min * Tr)) continue;
    if (STEP == 0) {
      atomicAdd(cnt + v.x, 1ull);
    } else {
      const int64_t pos = rowoff[v.x] + (int64_t)atomicAdd(cnt + v.x, 1ull);
      pat[pos] = v.y;
      xv[pos] = P / Tr / new_scaling[v.y];
    }
  }
}

// ------------------------------------------------------ rotation chunks --
// A maximize over rotation chunks holds Y for one chunk at a time.  After
// each chunk the running lse (the combine over the tile partials of the
// chunks so far) is a lower bound of the final one, so an entry whose P under
// it is below list_min stays below it: the chunk's row-sum sweep keeps the
// entries at or above it (rotation, pattern and y), and after the last chunk,
// whose combine covers every tile, the lse is final.

// LL of a candidate from its stored y (poisson: y; gaussian: C), in FP64.
__device__ __forceinline__ double cand_ll(const RespArgs& a, int64_t r, int64_t p, float y) {
  if (a.poisson) return (double)y;
  const double phi = a.scaling[p];
  return fma((double)y, 2.0 * a.gauss_inv / phi,
             -a.patstat[p] / (phi * phi) * a.gauss_inv - a.rowstat[r] * a.gauss_inv);
}

// Pv[e] = exp(LL - lse_p) as probs_from forms it; T64[r] += Pv[e].
__global__ void cand_finish_kernel(const RespArgs a, int64_t n, float* Pv, double* T64) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int2 v = a.list_rp[e];
    const double ll = cand_ll(a, v.x, v.y, a.list_P[e]);
    const float P = expf((float)(ll - a.lse[v.y]));
    Pv[e] = P;
    atomicAdd(T64 + v.x, (double)P);
  }
}

__global__ void T_from64_kernel(const double* T64, int64_t R, float* T) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) T[r] = (float)T64[r];
}

__global__ void cand_scatter_kernel(const int2* rp, const float* Pv, int64_t n, int64_t N,
                                    float* P) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int2 v = rp[e];
    P[(int64_t)v.x * N + v.y] = Pv[e];
  }
}

// one block per requested column
__global__ void cand_columns_kernel(const int2* rp, const float* Pv, int64_t n,
                                    const int64_t* cols, int64_t ncols, float* out) {
  const int64_t a = blockIdx.x, p = cols[a];
  for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
    const int2 v = rp[e];
    if (v.y == p) out[(int64_t)v.x * ncols + a] = Pv[e];
  }
}

// Total order of doubles as unsigned integers.
__device__ __forceinline__ unsigned long long ordered_bits(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// STEP 0: key[p] = max over the pattern's candidates of LL; STEP 1: best[p]
// = the lowest rotation whose LL is that maximum.
template <int STEP>
__global__ void cand_argmax_kernel(const RespArgs a, int64_t n, unsigned long long* key,
                                   int32_t* best) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int2 v = a.list_rp[e];
    const unsigned long long k = ordered_bits(cand_ll(a, v.x, v.y, a.list_P[e]));
    if (STEP == 0)
      atomicMax(key + v.y, k);
    else if (k == key[v.y])
      atomicMin(best + v.y, v.x);
  }
}

// bestp[p] = exp(max LL - lse_p); a pattern without candidates gets -1, 0.
__global__ void cand_bestp_kernel(const RespArgs a, const unsigned long long* key, int32_t* best,
                                  float* bestp) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.N) return;
  const unsigned long long k = key[p];
  if (k == 0) {
    best[p] = -1;
    bestp[p] = 0.0f;
    return;
  }
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  bestp[p] = (float)exp(__longlong_as_double((long long)b) - a.lse[p]);
}

__global__ void cand_cells_kernel(const int2* rp, const float* Pv, int64_t n, const int32_t* cell,
                                  int C, double* acc) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int2 v = rp[e];
    atomicAdd(acc + (int64_t)v.y * C + cell[v.x], (double)Pv[e]);
  }
}

__global__ void cells_out_kernel(const double* acc, int64_t count, int take_log, float* t) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double v = acc[i];
  t[i] = take_log ? (v > 0.0 ? (float)log(v) : -INFINITY) : (float)v;
}

// --------------------------------------------- deterministic list order --
// The compaction appends entries in the order warps reach it.  For the
// deterministic mode they are sorted by (rotation, pattern) with a stable
// LSD radix sort, 8 bits per pass (pattern bits first): per tile of
// kSortTile entries the digit counts hist[digit][tile], one exclusive scan
// over them digit-major, then one warp per tile writes its entries in order
// (ranks within a warp's 32 entries by __match_any_sync).
constexpr int kSortTile = 1024;

__device__ __forceinline__ uint32_t sort_digit(int2 v, int field, int shift) {
  return ((uint32_t)(field ? v.x : v.y) >> shift) & 0xffu;
}

__global__ void radix_hist_kernel(const int2* rp, int64_t n, int field, int shift,
                                  int64_t ntiles, int64_t* hist) {
  __shared__ int cnt[256];
  const int64_t tile = blockIdx.x;
  for (int d = threadIdx.x; d < 256; d += blockDim.x) cnt[d] = 0;
  __syncthreads();
  const int64_t e0 = tile * kSortTile;
  for (int64_t e = e0 + threadIdx.x; e < n && e < e0 + kSortTile; e += blockDim.x)
    atomicAdd(&cnt[sort_digit(rp[e], field, shift)], 1);
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[(int64_t)d * ntiles + tile] = cnt[d];
}

__global__ void radix_scatter_kernel(const int2* rp, const float* v, int64_t n, int field,
                                     int shift, int64_t ntiles, const int64_t* off, int2* rp2,
                                     float* v2) {
  __shared__ int64_t base[256];
  const int64_t tile = blockIdx.x;
  const int lane = threadIdx.x;
  for (int d = lane; d < 256; d += 32) base[d] = off[(int64_t)d * ntiles + tile];
  __syncwarp();
  const int64_t e0 = tile * kSortTile;
  const int64_t e1 = e0 + kSortTile < n ? e0 + kSortTile : n;
  for (int64_t c = e0; c < e1; c += 32) {
    const int64_t e = c + lane;
    const unsigned active = __ballot_sync(0xffffffffu, e < e1);
    if (e < e1) {
      const int2 x = rp[e];
      const uint32_t d = sort_digit(x, field, shift);
      const unsigned peers = __match_any_sync(active, d);
      const int rank = __popc(peers & ((1u << lane) - 1u));
      const int64_t pos = base[d] + rank;
      rp2[pos] = x;
      v2[pos] = v[e];
      __syncwarp(active);
      // the group's last lane moves the digit's offset past the group
      if ((peers >> lane) == 1u) base[d] += __popc(peers);
    }
    __syncwarp();
  }
}

// Entries sorted by rotation: rowtot[r] = entries of row r (all, or those
// kept by the list filter P >= rel_min T_r, T_r > 0), flag[e] = kept.
__global__ void sorted_count_kernel(const int2* rp, const float* Pv, int64_t n, const float* T,
                                    float rel_min, int filter, unsigned long long* rowtot,
                                    int64_t* flag) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int2 v = rp[e];
    bool keep = true;
    if (filter) {
      const float Tr = T[v.x];
      keep = Tr > 0.0f && Pv[e] >= rel_min * Tr;
    }
    if (flag) flag[e] = keep ? 1 : 0;
    if (keep) atomicAdd(rowtot + v.x, 1ull);
  }
}

// T_r = sum of the row's sorted entries in order (FP64).
__global__ void sorted_T_kernel(const float* Pv, const int64_t* rowoff, int64_t R, float* T) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  double t = 0.0;
  for (int64_t e = rowoff[r]; e < rowoff[r + 1]; ++e) t += Pv[e];
  T[r] = (float)t;
}

// Kept entries to their list positions (the exclusive scan of flag).
__global__ void sorted_place_kernel(const int2* rp, const float* Pv, int64_t n, const float* T,
                                    const float* new_scaling, const int64_t* flag,
                                    const int64_t* pos, int32_t* pat, float* xv) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[e]) continue;
    const int2 v = rp[e];
    pat[pos[e]] = v.y;
    xv[pos[e]] = Pv[e] / T[v.x] / new_scaling[v.y];
  }
}

// Compress from the lists: one block per rotation.  U_r / T_r over the active
// pixels is accumulated in shared memory from the listed patterns' photon
// lists (x times each non-zero count), then inserted exactly as the dense
// contraction's epilogue does (EpiCmp).
__global__ void __launch_bounds__(256) list_compress_kernel(const ListCmpArgs a) {
  extern __shared__ float Us[];  // [npa]
  const int64_t r = blockIdx.x;
  const CmpEpiArgs& e = a.e;
  if (a.gate_count && *a.gate_count > (unsigned long long)a.gate_cap) return;
  const float T = e.T[r];
  if (!((e.Tskip ? e.Tskip[r] : T) > 1e-10f) || !(T > 0.0f)) return;  // emc_atomic.cu:128
  for (int64_t j = threadIdx.x; j < e.npa; j += blockDim.x) Us[j] = 0.0f;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (a.ordered) {
    // the listed patterns in list order by one warp: a pattern's photons lie
    // on distinct pixels, so each pixel sums its terms in that order
    if (w == 0)
      for (int64_t q = a.rowoff[r]; q < a.rowoff[r + 1]; ++q) {
        const int64_t p = a.pat[q];
        const float x = a.xv[q];
        for (int64_t t = a.kptr[p] + lane; t < a.kptr[p + 1]; t += 32)
          Us[a.kidx[t]] += x * a.kval[t];
        __syncwarp();
      }
  } else {
    for (int64_t q = a.rowoff[r] + w; q < a.rowoff[r + 1]; q += blockDim.x >> 5) {
      const int64_t p = a.pat[q];
      const float x = a.xv[q];
      for (int64_t t = a.kptr[p] + lane; t < a.kptr[p + 1]; t += 32)
        atomicAdd(&Us[a.kidx[t]], x * a.kval[t]);
    }
  }
  __syncthreads();
  const float wT = e.rotw[r] * T;
  float m[9];
  emc_voxel::rotation_matrix(e.quat + 4 * r, m);
  for (int64_t j = threadIdx.x; j < e.npa; j += blockDim.x) {
    if (e.ins[j] != 1) continue;
    float u[3];
    emc_voxel::position(m, e.side, e.cx[j], e.cy[j], e.cz[j], u);
    const float val = Us[j] * wT;
    if (e.interp == 0) {
      int64_t vox;
      if (emc_voxel::nearest(u, e.side, 0, &vox)) insert_add(e, vox, val, wT);
    } else {
#pragma unroll
      for (int cc = 0; cc < 8; ++cc) {
        int64_t vox;
        float wc;
        if (!emc_voxel::trilinear_corner(u, e.side, cc, &vox, &wc) || wc == 0.0f) continue;
        insert_add(e, vox, wc * val, wc * wT);
      }
    }
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

// Most probable rotation of every pattern from Y: best[p] = argmax_r LL_rp,
// bestp[p] = exp(LL - lse_p); 32 patterns per block, 8 warps split R.
__global__ void __launch_bounds__(256) resp_argmax_kernel(const RespArgs a, int32_t* best,
                                                          float* bestp) {
  __shared__ double sv[8][32];
  __shared__ int32_t si[8][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t p = (int64_t)blockIdx.x * 32 + lane;
  const LLFromY f = make_llf(a, p < a.N ? p : 0);
  double bv = -INFINITY;
  int32_t bi = -1;
  if (p < a.N)
    for (int64_t r = w; r < a.R; r += 8) {
      const double rs = a.poisson ? 0.0 : a.rowstat[r] * a.gauss_inv;
      const double v = f(a.Y[r * a.ldY + p], rs);
      if (v > bv) {
        bv = v;
        bi = (int32_t)r;
      }
    }
  sv[w][lane] = bv;
  si[w][lane] = bi;
  __syncthreads();
  if (w == 0 && p < a.N) {
    for (int k = 1; k < 8; ++k)
      if (sv[k][lane] > bv || (sv[k][lane] == bv && si[k][lane] >= 0 && si[k][lane] < bi)) {
        bv = sv[k][lane];
        bi = si[k][lane];
      }
    best[p] = bi;
    bestp[p] = (float)exp(bv - a.lse[p]);
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

cudaError_t launch_wait_probe(TcStatus* status, uint64_t limit_ns, cudaStream_t st) {
  wait_probe_kernel<<<1, 32, 0, st>>>(status, limit_ns);
  return cudaGetLastError();
}

bool tc_encode_2d(CUtensorMap* tm, const void* base, uint64_t inner, uint64_t rows,
                  uint32_t box_rows, uint32_t box_inner) {
  return tc_encode_2d_strided(tm, base, inner, rows, inner, box_rows, box_inner);
}

bool tc_encode_2d_strided(CUtensorMap* tm, const void* base, uint64_t inner, uint64_t rows,
                          uint64_t ld, uint32_t box_rows, uint32_t box_inner) {
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
  const cuuint64_t strides[1] = {ld * 2};
  if (box_inner != 64 && box_inner != 32) return false;
  if (ld < inner || (ld * 2) % 16 != 0) return false;
  const cuuint32_t box[2] = {box_inner, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(base), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            box_inner == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_maximize_tc(const CUtensorMap& tmK, const CUtensorMap& tmBhi,
                               const CUtensorMap& tmBlo, int64_t Mpad, int64_t Rpad,
                               int64_t Kpad, const MaxEpiArgs& e, TcStatus* status, int num_sms,
                               cudaStream_t st, int raster) {
  EpiMax epi;
  epi.a = e;
  // rows = patterns (counts, 8 KB per stage), columns = rotations (hi and lo,
  // 2 x 16 KB); pattern tiles are the inner index, so the CTAs in flight share
  // each rotation tile in L2.  K-steps of 32 (64-byte rows) keep five 40 KB
  // stages in flight.
  return run_gemm<1, 2, 5, true, kMaximizeBK>(one_set(tmK, tmK, tmBhi, tmBlo), Mpad / BM, Rpad / BN,
                                              Kpad / kMaximizeBK, epi, status, num_sms, st,
                                              raster);
}

cudaError_t launch_maximize_pair_tc(const CUtensorMap& tmK, const CUtensorMap& tmBhi,
                                    const CUtensorMap& tmBlo, int64_t Mpad, int64_t Rpad,
                                    int64_t Kpad, const MaxEpiArgs& e, TcStatus* status,
                                    int num_sms, cudaStream_t st, int raster) {
  EpiMaxT<8> epi;  // two epilogue warps per TMEM lane quarter
  epi.a = e;
  // 256-pattern pair tiles (the last may reach past Mpad: zero-filled by TMA,
  // masked by the epilogue), 64-wide K-steps
  return run_pair<1, 2, true>(one_set(tmK, tmK, tmBhi, tmBlo), (Mpad + 255) / 256, Rpad / BN,
                             Kpad / kPairBK, epi, status, num_sms, st, raster);
}

cudaError_t launch_compress_pair_tc(const CUtensorMap& tmPhi, const CUtensorMap& tmPlo,
                                    const CUtensorMap& tmKt, int64_t Rpad, int64_t Ppad,
                                    int64_t Npad, const CmpEpiArgs& e, TcStatus* status,
                                    int num_sms, cudaStream_t st, int raster) {
  EpiCmp epi;
  epi.a = e;
  // 256-rotation pair tiles (Rpad is a multiple of 256), pixel tiles inner
  return run_pair<2, 1, false>(one_set(tmPhi, tmPlo, tmKt, tmKt), Rpad / 256, Ppad / BN,
                               Npad / kPairBK, epi, status, num_sms, st, raster);
}

cudaError_t launch_compress_tc(const CUtensorMap& tmPhi, const CUtensorMap& tmPlo,
                               const CUtensorMap& tmKt, int64_t Rpad, int64_t Ppad, int64_t Npad,
                               const CmpEpiArgs& e, TcStatus* status, int num_sms,
                               cudaStream_t st, int raster) {
  EpiCmp epi;
  epi.a = e;
  // pixel tiles are the inner index: CTAs in flight share the P' tiles
  return run_gemm<2, 1, 3, false, kCompressBK>(one_set(tmPhi, tmPlo, tmKt, tmKt), Rpad / BM, Ppad / BN,
                                               Npad / kCompressBK, epi, status, num_sms, st,
                                               raster);
}

cudaError_t launch_group_maximize_tc(const CUtensorMap& tmKg, const CUtensorMap& tmBhi,
                                     const CUtensorMap& tmBlo, int64_t n_tiles,
                                     const GMaxEpiArgs& e, TcStatus* status, int num_sms,
                                     cudaStream_t st) {
  EpiGMax epi;
  epi.a = e;
  return run_gemm<1, 2, 5, true, kMaximizeBK>(one_set(tmKg, tmKg, tmBhi, tmBlo), n_tiles, 1, 0, epi,
                                              status, num_sms, st);
}

cudaError_t launch_group_maximize_pair_tc(const CUtensorMap& tmKg, const CUtensorMap& tmBhi,
                                          const CUtensorMap& tmBlo, int64_t n_tiles,
                                          const GMaxEpiArgs& e, TcStatus* status, int num_sms,
                                          cudaStream_t st) {
  EpiGMaxPair epi;
  epi.a = e;
  return run_pair<1, 2, true>(one_set(tmKg, tmKg, tmBhi, tmBlo), n_tiles, 1, 0, epi, status,
                              num_sms, st, 1);
}

cudaError_t launch_group_compress_tc(const CUtensorMap& tmAhi, const CUtensorMap& tmAlo,
                                     const CUtensorMap& tmKg64, int64_t n_tiles,
                                     const GCmpEpiArgs& e, TcStatus* status, int num_sms,
                                     cudaStream_t st) {
  EpiGCmp epi;
  epi.a = e;
  return run_gemm<2, 1, 3, false, kCompressBK>(one_set(tmAhi, tmAlo, tmKg64, tmKg64), n_tiles, 1,
                                               0, epi, status, num_sms, st);
}

cudaError_t launch_batch_maximize_tc(const TmapSet<kMaxBatch>& maps, int64_t n_tiles,
                                     const BatchMaxArgs& e, TcStatus* status, int num_sms,
                                     cudaStream_t st) {
  EpiBatchMax epi;
  epi.a = e;
  return run_gemm<1, 2, 5, true, kMaximizeBK>(maps, n_tiles, 1, 0, epi, status, num_sms, st);
}

cudaError_t launch_batch_maximize_pair_tc(const TmapSet<kMaxBatch>& maps, int64_t n_tiles,
                                          const BatchMaxArgs& e, TcStatus* status, int num_sms,
                                          cudaStream_t st) {
  EpiBatchMaxPair epi;
  epi.a = e;
  return run_pair<1, 2, true>(maps, n_tiles, 1, 0, epi, status, num_sms, st, 1);
}

cudaError_t launch_batch_compress_pair_tc(const TmapSet<kMaxBatch>& maps, int64_t n_tiles,
                                          const BatchCmpArgs& e, TcStatus* status, int num_sms,
                                          cudaStream_t st) {
  EpiBatchCmpPair epi;
  epi.a = e;
  return run_pair<2, 1, false>(maps, n_tiles, 1, 0, epi, status, num_sms, st, 1);
}

cudaError_t launch_batch_compress_tc(const TmapSet<kMaxBatch>& maps, int64_t n_tiles,
                                     const BatchCmpArgs& e, TcStatus* status, int num_sms,
                                     cudaStream_t st) {
  EpiBatchCmp epi;
  epi.a = e;
  return run_gemm<2, 1, 3, false, kCompressBK>(maps, n_tiles, 1, 0, epi, status, num_sms, st);
}

cudaError_t launch_resp_rowsums(RespArgs& a, cudaStream_t st) {
  combine_kernel<<<(unsigned)((a.N + 255) / 256), 256, 0, st>>>(a);
  const int64_t nblk = (a.N + kSweepPatterns - 1) / kSweepPatterns;
  const int64_t rblk = (a.R + kSweepRows - 1) / kSweepRows;
  if (a.poisson)
    rowsum_kernel<true><<<dim3((unsigned)nblk, (unsigned)rblk), kSweepThreads, 0, st>>>(a);
  else
    rowsum_kernel<false><<<dim3((unsigned)nblk, (unsigned)rblk), kSweepThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_resp_write(RespArgs& a, cudaStream_t st) {
  const int64_t nblk = (a.N + kSweepPatterns - 1) / kSweepPatterns;
  const int64_t rblk = (a.R + kSweepRows - 1) / kSweepRows;
  const int64_t wblk = (a.ldP + kSweepPatterns - 1) / kSweepPatterns;
  const int64_t ntiles = wblk * rblk;
  const unsigned grid = (unsigned)(a.gate_count ? std::min<int64_t>(ntiles, 2048) : ntiles);
  if (a.poisson)
    write_kernel<true><<<grid, kSweepThreads, 0, st>>>(a, nblk, wblk, ntiles);
  else
    write_kernel<false><<<grid, kSweepThreads, 0, st>>>(a, nblk, wblk, ntiles);
  return cudaGetLastError();
}

cudaError_t launch_resp_pass(RespArgs& a, cudaStream_t st) {
  cudaError_t e = launch_resp_rowsums(a, st);
  return e == cudaSuccess ? launch_resp_write(a, st) : e;
}

int64_t resp_list_blocks(int64_t N) { return (N + kSweepPatterns - 1) / kSweepPatterns; }

cudaError_t launch_list_rowscan(const int64_t* rowtot, int64_t R, int64_t* rowoff,
                                cudaStream_t st) {
  list_rowscan_kernel<<<1, 1024, 0, st>>>(rowtot, R, rowoff);
  return cudaGetLastError();
}

cudaError_t launch_list_from_compact(RespArgs& a, int64_t n, float rel_min, int64_t* rowtot,
                                     int64_t* cursor, int64_t* rowoff, int32_t* pat, float* xv,
                                     cudaStream_t st, const unsigned long long* n_dev) {
  const int64_t nblk = resp_list_blocks(a.N);
  finish_T_kernel<<<(unsigned)((a.R + 255) / 256), 256, 0, st>>>(a.Tpart, nblk, a.R, a.T);
  cudaError_t e = cudaMemsetAsync(rowtot, 0, sizeof(int64_t) * a.R, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(cursor, 0, sizeof(int64_t) * a.R, st);
  if (e != cudaSuccess) return e;
  const unsigned g = (unsigned)std::min<int64_t>((n + 255) / 256 + 1, 4096);
  compact_sort_kernel<0><<<g, 256, 0, st>>>(a.list_rp, a.list_P, n, a.T, a.new_scaling, rel_min,
                                            reinterpret_cast<unsigned long long*>(rowtot),
                                            nullptr, nullptr, nullptr, n_dev);
  list_rowscan_kernel<<<1, 1024, 0, st>>>(rowtot, a.R, rowoff);
  compact_sort_kernel<1><<<g, 256, 0, st>>>(a.list_rp, a.list_P, n, a.T, a.new_scaling, rel_min,
                                            reinterpret_cast<unsigned long long*>(cursor), rowoff,
                                            pat, xv, n_dev);
  return cudaGetLastError();
}

static unsigned grid_for(int64_t n) {
  return (unsigned)std::min<int64_t>((n + 255) / 256 + 1, 4096);
}

cudaError_t launch_cand_probs(const RespArgs& a, int64_t n, float* Pv, double* T64,
                              cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(T64, 0, sizeof(double) * a.R, st);
  if (e != cudaSuccess) return e;
  if (n > 0) cand_finish_kernel<<<grid_for(n), 256, 0, st>>>(a, n, Pv, T64);
  return cudaGetLastError();
}

cudaError_t launch_list_from_candidates(RespArgs& a, int64_t n, float rel_min, float* Pv,
                                        double* T64, int64_t* rowtot, int64_t* cursor,
                                        int64_t* rowoff, int32_t* pat, float* xv, cudaStream_t st) {
  cudaError_t e = launch_cand_probs(a, n, Pv, T64, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(rowtot, 0, sizeof(int64_t) * a.R, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(cursor, 0, sizeof(int64_t) * a.R, st);
  if (e != cudaSuccess) return e;
  const unsigned g = grid_for(n);
  T_from64_kernel<<<(unsigned)((a.R + 255) / 256), 256, 0, st>>>(T64, a.R, a.T);
  compact_sort_kernel<0><<<g, 256, 0, st>>>(a.list_rp, Pv, n, a.T, a.new_scaling, rel_min,
                                            reinterpret_cast<unsigned long long*>(rowtot),
                                            nullptr, nullptr, nullptr, nullptr);
  list_rowscan_kernel<<<1, 1024, 0, st>>>(rowtot, a.R, rowoff);
  compact_sort_kernel<1><<<g, 256, 0, st>>>(a.list_rp, Pv, n, a.T, a.new_scaling, rel_min,
                                            reinterpret_cast<unsigned long long*>(cursor), rowoff,
                                            pat, xv, nullptr);
  return cudaGetLastError();
}

int64_t scan_scratch(int64_t n) { return 2 * ((n + kScanBlock - 1) / kScanBlock) + 2; }

// out[0..n] = exclusive prefix sums of in[0..n) (out[n] = total); scratch
// [scan_scratch(n)].
static cudaError_t scan_i64(const int64_t* in, int64_t n, int64_t* out, int64_t* scratch,
                            cudaStream_t st) {
  const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
  if (nb == 0) return cudaMemsetAsync(out, 0, sizeof(int64_t), st);
  scan_totals_kernel<<<(unsigned)nb, 1024, 0, st>>>(in, n, scratch);
  list_rowscan_kernel<<<1, 1024, 0, st>>>(scratch, nb, scratch + nb);
  scan_apply_kernel<<<(unsigned)nb, 1024, 0, st>>>(in, n, scratch + nb, out);
  return cudaGetLastError();
}

int64_t sort_hist_size(int64_t n) {
  const int64_t hn = 256 * ((n + kSortTile - 1) / kSortTile);
  return 2 * hn + 1 + scan_scratch(hn);
}

cudaError_t launch_sort_entries(int2* rp, float* v, int64_t n, int64_t N, int64_t R, int2* rp2,
                                float* v2, int64_t* hist, cudaStream_t st) {
  if (n <= 1) return cudaSuccess;
  const int64_t ntiles = (n + kSortTile - 1) / kSortTile;
  const int64_t hn = 256 * ntiles;
  auto bits = [](int64_t m) {
    int b = 1;
    while (b < 31 && (int64_t(1) << b) < m) ++b;
    return b;
  };
  int2 *src = rp, *dst = rp2;
  float *vs = v, *vd = v2;
  for (int field = 0; field < 2; ++field) {
    const int nb = bits(field ? R : N);
    for (int shift = 0; shift < nb; shift += 8) {
      // counts in hist[0 .. hn), their exclusive offsets in hist[hn .. 2 hn]
      radix_hist_kernel<<<(unsigned)ntiles, 256, 0, st>>>(src, n, field, shift, ntiles, hist);
      cudaError_t e = scan_i64(hist, hn, hist + hn, hist + 2 * hn + 1, st);
      if (e != cudaSuccess) return e;
      radix_scatter_kernel<<<(unsigned)ntiles, 32, 0, st>>>(src, vs, n, field, shift, ntiles,
                                                            hist + hn, dst, vd);
      std::swap(src, dst);
      std::swap(vs, vd);
    }
  }
  if (src != rp) {
    cudaError_t e = cudaMemcpyAsync(rp, src, sizeof(int2) * n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v, vs, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

cudaError_t launch_T_from_sorted(const int2* rp, const float* Pv, int64_t n, int64_t R,
                                 int64_t* rowtot, int64_t* rowoff, float* T, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(rowtot, 0, sizeof(int64_t) * R, st);
  if (e != cudaSuccess) return e;
  if (n > 0)
    sorted_count_kernel<<<grid_for(n), 256, 0, st>>>(rp, Pv, n, nullptr, 0.0f, 0,
                                                     reinterpret_cast<unsigned long long*>(rowtot),
                                                     nullptr);
  list_rowscan_kernel<<<1, 1024, 0, st>>>(rowtot, R, rowoff);
  sorted_T_kernel<<<(unsigned)((R + 255) / 256), 256, 0, st>>>(Pv, rowoff, R, T);
  return cudaGetLastError();
}

cudaError_t launch_list_from_sorted(const int2* rp, const float* Pv, int64_t n, int64_t R,
                                    const float* T, const float* new_scaling, float rel_min,
                                    int64_t* rowtot, int64_t* rowoff, int64_t* flag,
                                    int32_t* pat, float* xv, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(rowtot, 0, sizeof(int64_t) * R, st);
  if (e != cudaSuccess) return e;
  if (n > 0)
    sorted_count_kernel<<<grid_for(n), 256, 0, st>>>(rp, Pv, n, T, rel_min, 1,
                                                     reinterpret_cast<unsigned long long*>(rowtot),
                                                     flag);
  list_rowscan_kernel<<<1, 1024, 0, st>>>(rowtot, R, rowoff);
  if (n > 0) {
    // positions: the exclusive scan of the flags, in flag[n + 1 ..]
    e = scan_i64(flag, n, flag + n + 1, flag + 2 * n + 2, st);
    if (e != cudaSuccess) return e;
    sorted_place_kernel<<<grid_for(n), 256, 0, st>>>(rp, Pv, n, T, new_scaling, flag,
                                                     flag + n + 1, pat, xv);
  }
  return cudaGetLastError();
}

cudaError_t launch_finish_T(const float* Tpart, int64_t N, int64_t R, float* T, cudaStream_t st) {
  finish_T_kernel<<<(unsigned)((R + 255) / 256), 256, 0, st>>>(Tpart, resp_list_blocks(N), R, T);
  return cudaGetLastError();
}

cudaError_t launch_cand_scatter(const int2* rp, const float* Pv, int64_t n, int64_t N, float* P,
                                cudaStream_t st) {
  if (n > 0) cand_scatter_kernel<<<grid_for(n), 256, 0, st>>>(rp, Pv, n, N, P);
  return cudaGetLastError();
}

cudaError_t launch_cand_columns(const int2* rp, const float* Pv, int64_t n, const int64_t* cols,
                                int64_t ncols, float* out, cudaStream_t st) {
  if (n > 0 && ncols > 0)
    cand_columns_kernel<<<(unsigned)ncols, 256, 0, st>>>(rp, Pv, n, cols, ncols, out);
  return cudaGetLastError();
}

cudaError_t launch_cand_argmax(const RespArgs& a, int64_t n, unsigned long long* key,
                               int32_t* best, float* bestp, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(key, 0, sizeof(unsigned long long) * a.N, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(best, 0x7f, sizeof(int32_t) * a.N, st);
  if (e != cudaSuccess) return e;
  if (n > 0) {
    cand_argmax_kernel<0><<<grid_for(n), 256, 0, st>>>(a, n, key, best);
    cand_argmax_kernel<1><<<grid_for(n), 256, 0, st>>>(a, n, key, best);
  }
  cand_bestp_kernel<<<(unsigned)((a.N + 255) / 256), 256, 0, st>>>(a, key, best, bestp);
  return cudaGetLastError();
}

cudaError_t launch_cand_cells(const int2* rp, const float* Pv, int64_t n, const int32_t* cell,
                              int C, double* acc, cudaStream_t st) {
  if (n > 0) cand_cells_kernel<<<grid_for(n), 256, 0, st>>>(rp, Pv, n, cell, C, acc);
  return cudaGetLastError();
}

cudaError_t launch_cells_out(const double* acc, int64_t count, int take_log, float* t,
                             cudaStream_t st) {
  if (count > 0)
    cells_out_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(acc, count, take_log, t);
  return cudaGetLastError();
}

cudaError_t launch_list_compress(const ListCmpArgs& a, cudaStream_t st) {
  const size_t smem = sizeof(float) * (size_t)a.e.npa;
  cudaError_t e = cudaFuncSetAttribute(list_compress_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (a.e.R > 0) list_compress_kernel<<<(unsigned)a.e.R, 256, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_resp_export(const RespArgs& a, float* P, cudaStream_t st) {
  dim3 grid((unsigned)((a.N + 255) / 256), (unsigned)(a.R < 4096 ? a.R : 4096));
  export_kernel<<<grid, 256, 0, st>>>(a, P);
  return cudaGetLastError();
}

cudaError_t launch_resp_argmax(const RespArgs& a, int32_t* best, float* bestp, cudaStream_t st) {
  resp_argmax_kernel<<<(unsigned)((a.N + 31) / 32), 256, 0, st>>>(a, best, bestp);
  return cudaGetLastError();
}

cudaError_t launch_pack_patterns(const float* K, int64_t N, int64_t npa, int64_t Npad,
                                 int64_t Ppad, __half* Kh, __half* Kt, int* bad, cudaStream_t st) {
  dim3 grid((unsigned)((Ppad + 31) / 32), (unsigned)((Npad + 31) / 32));
  pack_kernel<<<grid, dim3(32, 8), 0, st>>>(K, N, npa, Npad, Ppad, Kh, Kt, bad);
  return cudaGetLastError();
}

}  // namespace emc
