// FP64 tensor-core tile engine for complex double (cuDoubleComplex), sm_100a.
//
// The products of the complex path (zherk / zgemm2 / ztrmm2 steps of ?potrf,
// ?trtri, ?lauum) run on the same warp-level DMMA instruction as the real FP64
// engine (mma.sync.aligned.m16n8k4.row.col.f64), as four real products per complex
// multiply-add ("4M"):
//     Re C += Re a Re b - Im a' Im b'        Im C += Re a Im b' + Im a' Re b
// with a' = conj(a) / b' = conj(b) when the view is conjugated.  The signs are
// applied to the fragments (sign-bit flips on the integer pipe), so every MMA is a
// plain accumulate.  Each output keeps two FP64 accumulators (Re, Im).
//
// Tiles: 64 x 64 complex outputs per CTA, four warps of 32 x 32 (2 m16 x 4 n8 blocks,
// Re and Im: 64 accumulators per thread, as in the real engine), or, for products with
// k < 1024, 32 x 64 with warps of 16 x 32 (three CTAs per SM).  A stage holds 8
// complex k of both operands (2 x 8 KB), staged by TMA (cp.async.bulk.tensor.2d,
// 128-byte swizzle, no multicast) as FP64 pairs into a 4-stage mbarrier ring; two
// CTAs share an SM.  Thread 0 issues the copies; each warp releases a stage on its
// "empty" mbarrier, and thread 0, after consuming item q, refills the stage of item
// q - 1 (no CTA-wide barrier in the k loop).
//
// Shared memory, one stage and operand (views as in gemm.cuh, complex elements):
//   layout R (rows contiguous): 8 boxes of 8 complex rows x 8 k; a k-row of a box is
//            128 bytes (8 complex = 16 doubles), its 16-byte chunks (one complex each)
//            XOR-swizzled by (k & 7);
//   layout K (k contiguous):    64 rows of 8 complex k (128 bytes), chunks swizzled by
//            (row & 7).
// MMA step s (0, 1) of a stage, lane slot t holds complex k = 2t + s; fragment rows
// and columns are not permuted.  In both layouts the eight lanes of a quarter warp
// (g in {2q, 2q + 1}, t = 0..3) read chunks (2t + s) ^ g: eight distinct 16-byte
// chunks, so the 128-bit fragment loads are bank-conflict free.
#pragma once
#include <cuComplex.h>
#include <cuda.h>
#include <stdint.h>
#include "dmma.cuh"

namespace cuchol {
namespace zmma {

constexpr int BN = 64, BK = 8;                            // complex elements
constexpr int WARPS = 4;                                  // 2 x 2 warps of (16 MB) x 32
constexpr int THREADS = WARPS * 32;
constexpr int B_STAGE = BN * BK * 16;                     // 8 KB

// A tile shape: MB m16 blocks per warp, BM = 32 MB rows per CTA (MB = 2: 64 x 64 tiles,
// two CTAs per SM; MB = 1: 32 x 64 tiles, half the accumulators, three CTAs per SM).
template <int MB>
struct Shape {
  static constexpr int BM = 32 * MB;
  static constexpr int STAGES = 4;
  static constexpr int MIN_CTAS = MB == 2 ? 2 : 3;
  static constexpr int A_STAGE = BM * BK * 16;            // 8 KB (MB = 2) or 4 KB
  static constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;   // + 1 KB alignment slack
};
constexpr int BOX = 1024;                                 // layout R box: 8 rows x 8 k

using dmma::LAYOUT_K;
using dmma::LAYOUT_R;

struct Params {
  cuDoubleComplex* c; long long c_rs, c_cs;
  const cuDoubleComplex* cin; long long cin_rs, cin_cs;
  int m, n, k;
  cuDoubleComplex alpha, beta;
  int conj_a, conj_b;
  int tri_a, tri_b, unit_a, unit_b;
  int lower_only, real_diag;
  int tiles_m, tiles_n;
  int preload;      // alpha = +-1: accumulators start at beta * Cin
  int neg;          // alpha = -1 (with preload): the B fragments are negated
  int* err;         // set when a bounded wait gave up
};

// x with its sign bit XORed by `m` (0 or 0x80000000), on the integer pipe
__device__ __forceinline__ double flip(double x, uint32_t m) {
  return __hiloint2double(__double2hiint(x) ^ (int)m, __double2loint(x));
}

template <int L, int ROWS>
__device__ __forceinline__ void load_operand(const CUtensorMap* map, uint64_t* bar, unsigned char* dst, int r0,
                                             int k0) {
  if constexpr (L == LAYOUT_R) {
    // real view: 2 * rows x k doubles; a box is 16 doubles (8 complex rows) x 8 k
#pragma unroll
    for (int b = 0; b < ROWS / 8; ++b) dmma::tma_load_2d(map, bar, dst + b * BOX, 2 * (r0 + 8 * b), k0);
  } else {
    // real view: rows x 2k doubles; one box of 16 doubles (8 complex k) x ROWS rows
    dmma::tma_load_2d(map, bar, dst, 2 * k0, r0);
  }
}

// Fragment (Re, Im) of complex element (row, k) of a staged operand tile.
template <int L>
__device__ __forceinline__ double2 frag(const unsigned char* tile, int row, int k) {
  if constexpr (L == LAYOUT_R) {
    return *reinterpret_cast<const double2*>(tile + (row >> 3) * BOX + k * 128 + (((row & 7) ^ (k & 7)) << 4));
  } else {
    return *reinterpret_cast<const double2*>(tile + row * 128 + ((k ^ (row & 7)) << 4));
  }
}

// Triangular view: (row, k) outside the triangle reads zero, a unit diagonal one.
__device__ __forceinline__ double2 tri_mask(double2 v, int tri, int unit, int row, int k) {
  if (unit && row == k) return make_double2(1.0, 0.0);
  if (tri == TRI_LOWER && k > row) return make_double2(0.0, 0.0);
  if (tri == TRI_UPPER && k < row) return make_double2(0.0, 0.0);
  return v;
}

__device__ __forceinline__ cuDoubleComplex cmul(cuDoubleComplex a, cuDoubleComplex b) {
  return make_cuDoubleComplex(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

template <int LA, int LB, bool TRI, int MB>
__global__ void __launch_bounds__(THREADS, Shape<MB>::MIN_CTAS)
gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
            const __grid_constant__ Params P, const int* __restrict__ abort_flag) {
  constexpr int BM = Shape<MB>::BM, STAGES = Shape<MB>::STAGES;
  constexpr int A_STAGE = Shape<MB>::A_STAGE, STAGE_BYTES = Shape<MB>::STAGE_BYTES;
  if (cta_aborted(abort_flag)) return;
  const int ntiles = P.tiles_m * P.tiles_n;
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
      dmma::mbar_init(&full_bar[s], 1);
      dmma::mbar_init(&empty_bar[s], WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  // thread 0 fills the ring in consumption order: item q -> stage q % STAGES
  int p_tile = (int)blockIdx.x - (int)gridDim.x, p_kt = 0, p_KT = 0, p_i0 = 0, p_j0 = 0, p_kbase = 0;
  long long issued = 0, consumed = 0;
  auto produce = [&]() -> bool {
    while (p_kt >= p_KT) {
      p_tile += gridDim.x;
      if (p_tile >= ntiles) return false;
      p_kt = 0;
      if (!tile_range(p_tile, p_i0, p_j0, p_kbase, p_KT)) p_KT = 0;
    }
    const int s = (int)(issued % STAGES);
    unsigned char* st = smem + s * STAGE_BYTES;
    dmma::mbar_expect_tx(&full_bar[s], STAGE_BYTES);
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
      if (!dmma::mbar_wait(&empty_bar[old % STAGES], (unsigned)((old / STAGES) & 1))) return false;
      more = produce();
    }
    return true;
  };

  const int wm = warp & 1, wn = warp >> 1;
  const int g = lane >> 2, t = lane & 3;
  constexpr uint32_t SIGN = 0x80000000u;
  // sign masks: Im a' = Im a (conj_a: -); B real part (neg: -); Im b' (conj_b xor neg)
  const uint32_t m_ai = P.conj_a ? SIGN : 0u;
  const uint32_t m_br = P.neg ? SIGN : 0u;
  const uint32_t m_bi = ((P.conj_b != 0) != (P.neg != 0)) ? SIGN : 0u;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int i0, j0, kbase, KT;
    if (!tile_range(tile, i0, j0, kbase, KT)) continue;
    // acc[mb][nb8][e]: Re (accr) and Im (acci) of row wrow + mb*16 + g (+8 for e >= 2),
    // column wcol + nb8*8 + 2t + (e & 1)
    double accr[MB][4][4], acci[MB][4][4];
#pragma unroll
    for (int a = 0; a < MB; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int c = 0; c < 4; ++c) accr[a][b][c] = acci[a][b][c] = 0.0;
    const int wrow = i0 + wm * (16 * MB), wcol = j0 + wn * 32;
    if (P.preload && P.cin != nullptr) {
#pragma unroll
      for (int mb = 0; mb < MB; ++mb)
#pragma unroll
        for (int nb8 = 0; nb8 < 4; ++nb8)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int row = wrow + mb * 16 + g + (e >> 1) * 8;
            const int col = wcol + nb8 * 8 + 2 * t + (e & 1);
            if (row < P.m && col < P.n && (!P.lower_only || row >= col)) {
              const cuDoubleComplex v = cmul(P.beta, P.cin[row * P.cin_rs + (long long)col * P.cin_cs]);
              accr[mb][nb8][e] = v.x;
              acci[mb][nb8][e] = v.y;
            }
          }
    }
    for (int kt = 0; kt < KT; ++kt, ++consumed) {
      const int s = (int)(consumed % STAGES);
      // bounded wait, its outcome made warp-uniform
      if (!__all_sync(0xffffffffu, dmma::mbar_wait(&full_bar[s], (unsigned)((consumed / STAGES) & 1)))) {
        ok = false;
        break;
      }
      {
        const unsigned char* As = smem + s * STAGE_BYTES;
        const unsigned char* Bs = As + A_STAGE;
        const int ks = kbase + kt * BK;
        // k blocks that reach the diagonal of a triangular view (its unit diagonal too)
        const bool mask_a = TRI && ((P.tri_a == TRI_LOWER && ks + BK - 1 >= wrow) ||
                                    (P.tri_a == TRI_UPPER && ks <= wrow + 16 * MB - 1));
        const bool mask_b = TRI && ((P.tri_b == TRI_LOWER && ks + BK - 1 >= wcol) ||
                                    (P.tri_b == TRI_UPPER && ks <= wcol + 31));
#pragma unroll
        for (int s2 = 0; s2 < 2; ++s2) {
          const int k = 2 * t + s2;
          // B fragments: (Re b, Im b', -Im b') of column g of each n8 block at k
          double br[4], bi[4], nbi[4];
#pragma unroll
          for (int nb8 = 0; nb8 < 4; ++nb8) {
            const int c = wn * 32 + nb8 * 8 + g;
            double2 v = frag<LB>(Bs, c, k);
            if (mask_b) v = tri_mask(v, P.tri_b, P.unit_b, j0 + c, ks + k);
            br[nb8] = flip(v.x, m_br);
            bi[nb8] = flip(v.y, m_bi);
            nbi[nb8] = flip(v.y, m_bi ^ SIGN);
          }
          // A fragments: rows g and g + 8 of each m16 block (Re a, Im a')
          double ar[MB][2], ai[MB][2];
#pragma unroll
          for (int mb = 0; mb < MB; ++mb) {
            const int r0 = wm * (16 * MB) + mb * 16 + g;
            double2 a0 = frag<LA>(As, r0, k), a1 = frag<LA>(As, r0 + 8, k);
            if (mask_a) {
              a0 = tri_mask(a0, P.tri_a, P.unit_a, i0 + r0, ks + k);
              a1 = tri_mask(a1, P.tri_a, P.unit_a, i0 + r0 + 8, ks + k);
            }
            ar[mb][0] = a0.x; ar[mb][1] = a1.x;
            ai[mb][0] = flip(a0.y, m_ai); ai[mb][1] = flip(a1.y, m_ai);
          }
          // 16 independent accumulator chains; each chain's two MMAs of this step are
          // 16 MMAs apart
#pragma unroll
          for (int mb = 0; mb < MB; ++mb)
#pragma unroll
            for (int nb8 = 0; nb8 < 4; ++nb8) {
              dmma::dmma_16x8x4(accr[mb][nb8], ar[mb][0], ar[mb][1], br[nb8]);
              dmma::dmma_16x8x4(acci[mb][nb8], ar[mb][0], ar[mb][1], bi[nb8]);
            }
#pragma unroll
          for (int mb = 0; mb < MB; ++mb)
#pragma unroll
            for (int nb8 = 0; nb8 < 4; ++nb8) {
              dmma::dmma_16x8x4(accr[mb][nb8], ai[mb][0], ai[mb][1], nbi[nb8]);
              dmma::dmma_16x8x4(acci[mb][nb8], ai[mb][0], ai[mb][1], br[nb8]);
            }
        }
      }
      // this warp is done with stage s
      __syncwarp();
      if (lane == 0) dmma::mbar_arrive(&empty_bar[s]);
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
      if (lane == 0) atomicExch(P.err, 3);
      if (threadIdx.x == 0)
        for (long long q = consumed; q < issued; ++q)
          dmma::mbar_wait(&full_bar[q % STAGES], (unsigned)((q / STAGES) & 1));
      return;
    }

    // epilogue: preload -> C = acc; else C = alpha * acc + beta * Cin
    const bool has_cin = (P.cin != nullptr) && !P.preload;
#pragma unroll
    for (int mb = 0; mb < MB; ++mb)
#pragma unroll
      for (int nb8 = 0; nb8 < 4; ++nb8)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int row = wrow + mb * 16 + g + (e >> 1) * 8;
          const int col = wcol + nb8 * 8 + 2 * t + (e & 1);
          if (row < P.m && col < P.n && (!P.lower_only || row >= col)) {
            cuDoubleComplex v = make_cuDoubleComplex(accr[mb][nb8][e], acci[mb][nb8][e]);
            if (!P.preload) v = cmul(P.alpha, v);
            if (has_cin) {
              const cuDoubleComplex o = cmul(P.beta, P.cin[row * P.cin_rs + (long long)col * P.cin_cs]);
              v.x += o.x;
              v.y += o.y;
            }
            if (P.real_diag && row == col) v.y = 0.0;
            P.c[row * P.c_rs + (long long)col * P.c_cs] = v;
          }
        }
  }
}

}  // namespace zmma
}  // namespace cuchol
