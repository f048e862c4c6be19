// FP64 tensor-core tile engine for sm_100a (double precision).
//
// Blackwell's tcgen05.mma has no f64 kind, so FP64 products run on the warp-level
// DMMA instruction mma.sync.aligned.m16n8k4.row.col.f64 (measured on B200: 37.1
// TFLOP/s device-wide, the same rate as DFMA).  Operand tiles are staged into
// shared memory by TMA (cp.async.bulk.tensor.2d, 128-byte swizzle, no multicast)
// through a 4-stage ring: thread 0 issues the copies (completion tracked by one
// "full" mbarrier per stage), and the CTA's four warps (2 x 2) run the MMAs on a
// 128 x 64 tile (warps of 64 x 32, two CTAs per SM) or a 64 x 64 tile (warps of
// 32 x 32, three CTAs per SM).  No dedicated producer warp: it would not fit the
// register budget of several CTAs per SM.  No CTA-wide barrier in the k loop either:
// each warp releases a stage by arriving on its "empty" mbarrier, and thread 0, after
// consuming item q, refills the stage of item q - 1 (which the other warps have almost
// always released by then), so the warps drift freely within the ring.
//
// Problem form: the GemmProblem of gemm.cuh for T = double,
//     C(i, j) = alpha * sum_k Ahat(i, k) * Bhat(j, k) + beta * Cin(i, j),
// with each view either row-contiguous (layout R: Ahat(i, k) = a[i + k*ld]) or
// k-contiguous (layout K: Ahat(i, k) = a[i*ld + k]), 16-byte aligned with an even
// leading dimension, optionally triangular (masked in registers on the k blocks
// that cross the diagonal) and optionally lower-only in its output.
//
// Shared memory, one stage:
//   layout R: BROWS/16 boxes of 16 rows x 16 k; a k-row is 128 bytes (16 doubles of
//             consecutive rows), its 16-byte chunks XOR-swizzled by (k & 7);
//   layout K: BROWS rows of 16 k (128 bytes), chunks swizzled by (row & 7).
// The k order inside a 16-wide block is permuted: MMA step s (0..3), lane slot t
// holds k = (s>>1)*8 + 2t + (s&1), so a K-layout thread reads the k pair of two
// steps with one 128-bit load; an R-layout thread reads rows 2g, 2g+1 of one k with
// one 128-bit load.  In both layouts the eight lanes of a quarter warp touch eight
// distinct 16-byte chunks, so the fragment loads are bank-conflict free.
#pragma once
#include <cuda.h>
#include <stdint.h>
#include "gemm.cuh"

namespace cuchol {
namespace dmma {

constexpr int BN = 64, BK = 16;
constexpr int WARPS = 4;                           // 2 x 2 warps of (16 MB) x 32
constexpr int THREADS = WARPS * 32;
constexpr int B_STAGE = BN * BK * 8;               // 8 KB

// A tile shape: MB m16 blocks per warp, so BM = 32 MB rows per CTA (MB = 4: 128 x 64
// tiles, two CTAs per SM; MB = 2: 64 x 64 tiles, fewer registers, three CTAs per SM).
template <int MB>
struct Shape {
  static constexpr int BM = 32 * MB;
  static constexpr int STAGES = 4;
  static constexpr int MIN_CTAS = MB == 4 ? 2 : 3;  // CTAs per SM the registers allow
  static constexpr int A_STAGE = BM * BK * 8;       // 16 KB (MB = 4) or 8 KB
  static constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;   // + 1 KB alignment slack
};
constexpr unsigned kSpinLimit = 1u << 26;          // bounded mbarrier waits: at most 2^26 polls
constexpr unsigned long long kWaitNs = 1000000000ull;   // and at most one second

enum : int { LAYOUT_R = 0, LAYOUT_K = 1 };

struct Params {
  double* c; long long c_rs, c_cs;
  const double* cin; long long cin_rs, cin_cs;
  int m, n, k;
  double alpha, beta;
  int tri_a, tri_b, unit_a, unit_b;
  int lower_only;
  int tiles_m, tiles_n;
  int vec_ok;            // C / Cin 16-byte aligned along their unit stride, Cin == C
  int preload;           // alpha = +-1: accumulators start at beta*Cin (loaded before
                         // the k loop, so its latency hides under the TMA fill)
  int neg;               // alpha = -1 (with preload): B fragments are negated
  int* err;              // set when a bounded wait gave up
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait (polls and wall-clock time; a poll may suspend the thread for a while):
// false if it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 0; it < kSpinLimit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 15u) == 15u && global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}
__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void dmma_16x8x4(double (&d)[4], double a0, double a1, double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b));
}
__device__ __forceinline__ int fperm(int g) { return (g >> 1) | ((g & 1) << 2); }

// Issue the TMA copies of one operand tile (rows [r0, r0 + ROWS), k [k0, k0 + 16)).
template <int L, int ROWS>
__device__ __forceinline__ void load_operand(const CUtensorMap* map, uint64_t* bar, unsigned char* dst, int r0, int k0) {
  if constexpr (L == LAYOUT_R) {
#pragma unroll
    for (int b = 0; b < ROWS / 16; ++b) tma_load_2d(map, bar, dst + b * 2048, r0 + 16 * b, k0);
  } else {
    tma_load_2d(map, bar, dst, k0, r0);
  }
}

// Mask one loaded fragment value of a triangular view: (row, k) outside the
// triangle reads zero, a unit diagonal reads one.
__device__ __forceinline__ double tri_mask(double v, int tri, int unit, int row, int k) {
  if (unit && row == k) return 1.0;
  if (tri == TRI_LOWER && k > row) return 0.0;
  if (tri == TRI_UPPER && k < row) return 0.0;
  return v;
}

template <int LA, int LB, bool TRI, int MB>
__global__ void __launch_bounds__(THREADS, Shape<MB>::MIN_CTAS)
gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
            const __grid_constant__ Params P, const int* __restrict__ abort_flag) {
  constexpr int BM = Shape<MB>::BM, STAGES = Shape<MB>::STAGES;
  constexpr int A_STAGE = Shape<MB>::A_STAGE, STAGE_BYTES = Shape<MB>::STAGE_BYTES;
  if (cta_aborted(abort_flag)) return;
  // This CTA's tiles: blockIdx.x, blockIdx.x + gridDim.x, ...  The host picks the
  // grid so that a CTA handles several tiles: the TMA ring keeps streaming across
  // tile boundaries, while CTAs still retire often enough for other streams' kernels.
  const int ntiles = P.tiles_m * P.tiles_n;
  // rows i0, columns j0 and k range [kbase, kbase + KT*BK) of a tile (triangular
  // views limit it); false for a tile wholly above the diagonal of a lower-only output
  auto tile_range = [&](int tile, int& i0, int& j0, int& kbase, int& KT) -> bool {
    i0 = (tile / P.tiles_n) * BM;
    j0 = (tile % P.tiles_n) * BN;
    if (P.lower_only && j0 > i0 + BM - 1) return false;
    int kb = 0, ke = P.k;
    if (P.tri_a == TRI_LOWER) ke = min(ke, i0 + BM);
    if (P.tri_a == TRI_UPPER) kb = max(kb, i0);
    if (P.tri_b == TRI_LOWER) ke = min(ke, j0 + BN);
    if (P.tri_b == TRI_UPPER) kb = max(kb, j0);
    kbase = (kb / BK) * BK;
    KT = (ke > kbase) ? (ke - kbase + BK - 1) / BK : 0;
    return true;
  };

  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* smem =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ __align__(8) uint64_t empty_bar[STAGES];

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  // Thread 0 fills the ring in the order the tiles consume it: item q (the q-th
  // k block of this CTA, over all its tiles) goes to stage q % STAGES.
  int p_tile = (int)blockIdx.x - (int)gridDim.x, p_kt = 0, p_KT = 0, p_i0 = 0, p_j0 = 0, p_kbase = 0;
  long long issued = 0, consumed = 0;
  auto produce = [&]() -> bool {   // issue the next item; false when none is left
    while (p_kt >= p_KT) {
      p_tile += gridDim.x;
      if (p_tile >= ntiles) return false;
      p_kt = 0;
      if (!tile_range(p_tile, p_i0, p_j0, p_kbase, p_KT)) p_KT = 0;
    }
    const int s = (int)(issued % STAGES);
    unsigned char* st = smem + s * STAGE_BYTES;
    mbar_expect_tx(&full_bar[s], STAGE_BYTES);
    load_operand<LA, BM>(&mapA, &full_bar[s], st, p_i0, p_kbase + p_kt * BK);
    load_operand<LB, BN>(&mapB, &full_bar[s], st + A_STAGE, p_j0, p_kbase + p_kt * BK);
    ++p_kt;
    ++issued;
    return true;
  };
  bool more = true;   // thread 0: items are left to issue
  if (threadIdx.x == 0)
    for (int q = 0; q < STAGES && more; ++q) more = produce();
  // thread 0, after consuming item `consumed`: issue the items up to consumed - 1 +
  // STAGES, each into a stage whose previous item every warp has released (bounded
  // wait); false if a wait gave up
  auto refill = [&]() -> bool {
    while (more && issued < consumed + STAGES) {
      const long long old = issued - STAGES;
      if (!mbar_wait(&empty_bar[old % STAGES], (unsigned)((old / STAGES) & 1))) return false;
      more = produce();
    }
    return true;
  };

  // ---------------- MMA warps ----------------
  const int wm = warp & 1, wn = warp >> 1;
  const int g = lane >> 2, t = lane & 3;
  const int fg = fperm(g);
  // rows of this thread's A fragments inside an m16 block (a0, a1) and the column
  // of its B fragment inside an n8 block, per layout
  const int arow0 = (LA == LAYOUT_R) ? 2 * g : fg;
  const int arow1 = (LA == LAYOUT_R) ? 2 * g + 1 : fg + 8;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
  int i0, j0, kbase, KT;
  if (!tile_range(tile, i0, j0, kbase, KT)) continue;
  double acc[MB][4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;

  const int wrow = i0 + wm * (16 * MB), wcol = j0 + wn * 32;   // first row / column of the warp
  // acc[mb][nb8][e]: row = wrow + mb*16 + (e < 2 ? arow0 : arow1),
  //                  col = wcol + colof(nb8, e & 1)
  auto colof = [&](int nb8, int e1) -> int {
    if constexpr (LB == LAYOUT_R) return (nb8 >> 1) * 16 + 4 * t + 2 * e1 + (nb8 & 1);
    else return nb8 * 8 + t + 4 * e1;
  };
  const bool full_tile = (i0 + BM <= P.m) && (j0 + BN <= P.n) && (!P.lower_only || j0 + BN - 1 <= i0);
  const bool vec_rows = (LA == LAYOUT_R) && full_tile && P.vec_ok && P.c_rs == 1;
  const bool vec_cols = !vec_rows && (LB == LAYOUT_R) && full_tile && P.vec_ok && P.c_cs == 1;
  if (P.preload && P.cin != nullptr) {
    if (vec_rows) {
#pragma unroll
      for (int mb = 0; mb < MB; ++mb)
#pragma unroll
        for (int nb8 = 0; nb8 < 4; ++nb8)
#pragma unroll
          for (int e1 = 0; e1 < 2; ++e1) {
            const int row = wrow + mb * 16 + arow0, col = wcol + colof(nb8, e1);
            const double2 o = *reinterpret_cast<const double2*>(P.cin + row + (long long)col * P.cin_cs);
            acc[mb][nb8][e1] = P.beta * o.x;
            acc[mb][nb8][2 + e1] = P.beta * o.y;
          }
    } else if (vec_cols) {
#pragma unroll
      for (int mb = 0; mb < MB; ++mb)
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
          for (int p = 0; p < 2; ++p) {
            const int row = wrow + mb * 16 + (e < 2 ? arow0 : arow1);
            const int col = wcol + colof(2 * p, e & 1);
            const double2 o = *reinterpret_cast<const double2*>(P.cin + (long long)row * P.cin_rs + col);
            acc[mb][2 * p][e] = P.beta * o.x;
            acc[mb][2 * p + 1][e] = P.beta * o.y;
          }
    } else {
#pragma unroll
      for (int mb = 0; mb < MB; ++mb)
#pragma unroll
        for (int nb8 = 0; nb8 < 4; ++nb8)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int row = wrow + mb * 16 + (e < 2 ? arow0 : arow1);
            const int col = wcol + colof(nb8, e & 1);
            if (row < P.m && col < P.n && (!P.lower_only || row >= col))
              acc[mb][nb8][e] = P.beta * P.cin[row * P.cin_rs + (long long)col * P.cin_cs];
          }
    }
  }
  for (int kt = 0; kt < KT; ++kt, ++consumed) {
    const int s = (int)(consumed % STAGES);
    // bounded wait, its outcome made warp-uniform
    if (!__all_sync(0xffffffffu, mbar_wait(&full_bar[s], (unsigned)((consumed / STAGES) & 1)))) {
      ok = false;
      break;
    }
    {
    const unsigned char* As = smem + s * STAGE_BYTES;
    const unsigned char* Bs = As + A_STAGE;
    const int ks = kbase + kt * BK;
    const bool mask_a = TRI && ((P.tri_a == TRI_LOWER && ks + BK - 1 >= wrow) ||
                                (P.tri_a == TRI_UPPER && ks <= wrow + 16 * MB - 1));
    const bool mask_b = TRI && ((P.tri_b == TRI_LOWER && ks + BK - 1 >= wcol) ||
                                (P.tri_b == TRI_UPPER && ks <= wcol + 31));
#pragma unroll
    for (int q = 0; q < 2; ++q) {            // pairs of MMA k-steps (2q, 2q + 1)
      // B fragments for both steps of the pair
      double2 bv[4];
      if constexpr (LB == LAYOUT_R) {
        // bv[2p + s2] = (column 2g of box p, column 2g + 1) at the k of step 2q + s2
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          const unsigned char* box = Bs + (wn * 2 + p) * 2048;
#pragma unroll
          for (int s2 = 0; s2 < 2; ++s2) {
            const int k = q * 8 + 2 * t + s2;
            bv[2 * p + s2] = *reinterpret_cast<const double2*>(box + k * 128 + ((g ^ (k & 7)) << 4));
          }
        }
      } else {
        // bv[nb8] = (k of step 2q, k of step 2q + 1) at column fg of n8 block nb8
        const int ch = q * 4 + t;
#pragma unroll
        for (int nb8 = 0; nb8 < 4; ++nb8) {
          const int r = wn * 32 + nb8 * 8 + fg;
          bv[nb8] = *reinterpret_cast<const double2*>(Bs + r * 128 + ((ch ^ (r & 7)) << 4));
        }
      }
      if (mask_b) {
        if constexpr (LB == LAYOUT_R) {
#pragma unroll
          for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int s2 = 0; s2 < 2; ++s2) {
              const int k = ks + q * 8 + 2 * t + s2;
              const int cb = wcol + p * 16 + 2 * g;
              bv[2 * p + s2].x = tri_mask(bv[2 * p + s2].x, P.tri_b, P.unit_b, cb, k);
              bv[2 * p + s2].y = tri_mask(bv[2 * p + s2].y, P.tri_b, P.unit_b, cb + 1, k);
            }
        } else {
#pragma unroll
          for (int nb8 = 0; nb8 < 4; ++nb8) {
            const int k = ks + q * 8 + 2 * t;
            const int cb = wcol + nb8 * 8 + fg;
            bv[nb8].x = tri_mask(bv[nb8].x, P.tri_b, P.unit_b, cb, k);
            bv[nb8].y = tri_mask(bv[nb8].y, P.tri_b, P.unit_b, cb, k + 1);
          }
        }
      }
      if (P.neg) {   // after the triangle mask, so an implicit unit diagonal is negated too
#pragma unroll
        for (int v = 0; v < 4; ++v) bv[v] = make_double2(-bv[v].x, -bv[v].y);
      }
      if constexpr (LA == LAYOUT_R) {
        // step-major order: an accumulator is reused only after the 15 other MMAs
        // of the step, so back-to-back MMAs never depend on each other
#pragma unroll
        for (int s2 = 0; s2 < 2; ++s2) {
          const int k = q * 8 + 2 * t + s2;
          double2 av[MB];
#pragma unroll
          for (int mb = 0; mb < MB; ++mb) {
            const unsigned char* box = As + (wm * MB + mb) * 2048;
            av[mb] = *reinterpret_cast<const double2*>(box + k * 128 + ((g ^ (k & 7)) << 4));
            if (mask_a) {
              const int ra = wrow + mb * 16;
              av[mb].x = tri_mask(av[mb].x, P.tri_a, P.unit_a, ra + arow0, ks + k);
              av[mb].y = tri_mask(av[mb].y, P.tri_a, P.unit_a, ra + arow1, ks + k);
            }
          }
#pragma unroll
          for (int mb = 0; mb < MB; ++mb)
#pragma unroll
            for (int nb8 = 0; nb8 < 4; ++nb8) {
              double b;
              if constexpr (LB == LAYOUT_R) {
                const double2 v = bv[2 * (nb8 >> 1) + s2];
                b = (nb8 & 1) ? v.y : v.x;
              } else {
                b = s2 ? bv[nb8].y : bv[nb8].x;
              }
              dmma_16x8x4(acc[mb][nb8], av[mb].x, av[mb].y, b);
            }
        }
      } else {
#pragma unroll
      for (int mb = 0; mb < MB; ++mb) {
        // A fragments of m16 block mb: av[s2] = (row arow0, row arow1) at step 2q + s2
        double2 av[2];
        if constexpr (LA == LAYOUT_R) {
          const unsigned char* box = As + (wm * MB + mb) * 2048;
#pragma unroll
          for (int s2 = 0; s2 < 2; ++s2) {
            const int k = q * 8 + 2 * t + s2;
            av[s2] = *reinterpret_cast<const double2*>(box + k * 128 + ((g ^ (k & 7)) << 4));
          }
        } else {
          const int r0 = wm * (16 * MB) + mb * 16 + fg, r1 = r0 + 8;
          const int ch = q * 4 + t;
          const double2 x0 = *reinterpret_cast<const double2*>(As + r0 * 128 + ((ch ^ (r0 & 7)) << 4));
          const double2 x1 = *reinterpret_cast<const double2*>(As + r1 * 128 + ((ch ^ (r1 & 7)) << 4));
          av[0] = make_double2(x0.x, x1.x);
          av[1] = make_double2(x0.y, x1.y);
        }
        if (mask_a) {
#pragma unroll
          for (int s2 = 0; s2 < 2; ++s2) {
            const int k = ks + q * 8 + 2 * t + s2;
            const int ra = wrow + mb * 16;
            av[s2].x = tri_mask(av[s2].x, P.tri_a, P.unit_a, ra + arow0, k);
            av[s2].y = tri_mask(av[s2].y, P.tri_a, P.unit_a, ra + arow1, k);
          }
        }
#pragma unroll
        for (int s2 = 0; s2 < 2; ++s2)
#pragma unroll
          for (int nb8 = 0; nb8 < 4; ++nb8) {
            double b;
            if constexpr (LB == LAYOUT_R) {
              const double2 v = bv[2 * (nb8 >> 1) + s2];
              b = (nb8 & 1) ? v.y : v.x;
            } else {
              b = s2 ? bv[nb8].y : bv[nb8].x;
            }
            dmma_16x8x4(acc[mb][nb8], av[s2].x, av[s2].y, b);
          }
      }
    }
      }
    }
    // this warp is done with stage s
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty_bar[s]);
    if (warp == 0) {
      bool fine = true;
      if (lane == 0) fine = refill();
      if (!__shfl_sync(0xffffffffu, fine, 0)) {
        ok = false;
        ++consumed;
        break;
      }
    }
  }
  if (!ok) {
    // a wait gave up (the other warps' waits then give up too, within their
    // bounds): record it, and let thread 0 wait (bounded) for the copies it issued
    // before it exits
    if (lane == 0) atomicExch(P.err, 3);
    if (threadIdx.x == 0)
      for (long long q = consumed; q < issued; ++q) mbar_wait(&full_bar[q % STAGES], (unsigned)((q / STAGES) & 1));
    return;
  }

  // ---------------- epilogue ----------------
  // preload: C = acc; otherwise C = alpha * acc + beta * Cin
  const bool has_cin = (P.cin != nullptr) && !P.preload;
  const double alpha = P.preload ? 1.0 : P.alpha;
  if (vec_rows) {
    // column-major C: rows arow0 and arow0 + 1 are adjacent
#pragma unroll
    for (int mb = 0; mb < MB; ++mb)
#pragma unroll
      for (int nb8 = 0; nb8 < 4; ++nb8)
#pragma unroll
        for (int e1 = 0; e1 < 2; ++e1) {
          const int row = wrow + mb * 16 + arow0, col = wcol + colof(nb8, e1);
          double2* ptr = reinterpret_cast<double2*>(P.c + row + (long long)col * P.c_cs);
          double2 v = make_double2(alpha * acc[mb][nb8][e1], alpha * acc[mb][nb8][2 + e1]);
          if (has_cin) {
            const double2 o = *ptr;
            v.x = fma(P.beta, o.x, v.x);
            v.y = fma(P.beta, o.y, v.y);
          }
          *ptr = v;
        }
  } else if (vec_cols) {
    // row-contiguous C: the columns of n8 blocks 2p and 2p + 1 are adjacent
#pragma unroll
    for (int mb = 0; mb < MB; ++mb)
#pragma unroll
      for (int e = 0; e < 4; ++e)
#pragma unroll
        for (int p = 0; p < 2; ++p) {
          const int row = wrow + mb * 16 + (e < 2 ? arow0 : arow1);
          const int col = wcol + colof(2 * p, e & 1);
          double2* ptr = reinterpret_cast<double2*>(P.c + (long long)row * P.c_rs + col);
          double2 v = make_double2(alpha * acc[mb][2 * p][e], alpha * acc[mb][2 * p + 1][e]);
          if (has_cin) {
            const double2 o = *ptr;
            v.x = fma(P.beta, o.x, v.x);
            v.y = fma(P.beta, o.y, v.y);
          }
          *ptr = v;
        }
  } else {
#pragma unroll
    for (int mb = 0; mb < MB; ++mb)
#pragma unroll
      for (int nb8 = 0; nb8 < 4; ++nb8)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int row = wrow + mb * 16 + (e < 2 ? arow0 : arow1);
          const int col = wcol + colof(nb8, e & 1);
          if (row < P.m && col < P.n && (!P.lower_only || row >= col)) {
            double v = alpha * acc[mb][nb8][e];
            if (has_cin) v = fma(P.beta, P.cin[row * P.cin_rs + (long long)col * P.cin_cs], v);
            P.c[row * P.c_rs + (long long)col * P.c_cs] = v;
          }
        }
  }
  }   // tile loop
}

}  // namespace dmma
}  // namespace cuchol
