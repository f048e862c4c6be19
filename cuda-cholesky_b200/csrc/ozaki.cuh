// Ozaki-sliced FP64 trailing update on the tcgen05 INT8 tensor cores:
//
//     C(i, j) -= sum_l P(i, l) P(j, l),   i >= j,   C and P in FP64
//
// Each row i of P is scaled by a power of two 2^-e_i (|P(i, l)| 2^-e_i < 1) and cut into
// S signed 8-bit slices, P(i, l) = 2^e_i sum_t 2^-7t a_t(i, l) + (a remainder below
// 2^(e_i - 7S)), every step exact in FP64 (multiply by 2^7, take the integer part).
// The product then splits into integer products,
//     sum_l P(i, l) P(j, l) ~ 2^(e_i + e_j) sum_{t + u <= S + 1} 2^-7(t + u) (a_t a_u^T)(i, j),
// and every a_t a_u^T is computed exactly by kind::i8 MMAs with INT32 accumulation; the
// terms of one diagonal d = t + u share an accumulator (at most S k-long sums of
// |a| <= 127 products: S * k * 127^2 < 2^31 while S * k < 133144; the driver's
// k <= 2048 with S <= 8 stays eight times below).  The epilogue turns
// the S accumulators into FP64 (exact), scales them by 2^-7d (exact), sums them in
// FP64 and applies 2^(e_i + e_j): the only roundings are the final FP64 additions and
// the dropped terms t + u > S + 1, below 2^-7(S + 1) of |P_i| |P_j| k.
//
// One CTA computes a 128 x 128 tile of C.  TMEM holds 4 accumulators of 128 INT32
// columns (the whole 512 columns of the SM, one CTA per SM), so the diagonals run in
// two passes, d = 2..5 and d = 6..S+1, each folded into C:
//   * thread 0 streams the 128-row slice tiles A_t (k-major, 128-byte swizzle, one TMA
//     box per 128 k) through a 2-stage ring and, for each u of the pass, the slice tile
//     B_u through a 4-stage ring; a stage holds up to 256 of k, and a longer k (the
//     driver's 512) runs as consecutive 256-wide halves that accumulate into the same
//     TMEM accumulators, so one epilogue per pass serves the whole k;
//   * thread 32 issues tcgen05.mma.cta_group::1.kind::i8 (M = N = 128, K = 32) on
//     A_t x B_u into the accumulator of its diagonal and frees the stages with
//     tcgen05.commit;
//   * after each pass the 4 warps read the accumulators back (tcgen05.ld, warp w =
//     rows 32w..32w+31), combine them in FP64 registers and update C (FP64,
//     column-major).  (M = N = 128 MMAs run at about 2.5x the rate per multiply of
//     N = 64 ones on B200, which pays for the second pass over C.)
// Waits are bounded; a wait that gives up records an error word, the CTA waits
// (bounded) for its loads in flight, and the tensor memory is freed on every path.
#pragma once
#include "tc.cuh"

namespace cuchol {
namespace oz {

constexpr int BM = 128, BN = 128, THREADS = 128;
constexpr int KMAX = 256;                   // k of one ring stage (longer k: halves)
constexpr int MAX_SLICES = 8;
constexpr int NACC = 4;                     // accumulators per pass (4 x 128 TMEM columns)
constexpr int A_STAGES = 2, B_STAGES = 4;
constexpr int A_TILE = BM * KMAX, B_TILE = BN * KMAX;   // bytes (int8)
constexpr int SMEM_BYTES = A_STAGES * A_TILE + B_STAGES * B_TILE + 1024;

struct Params {
  double* c; long long crs, ccs;   // C(i, j) = c[i*crs + j*ccs] (a region whose corner is on the diagonal)
  int m, n, k;                  // C region m x n (m >= n), slice rows: m (A side), n (B side) from row0
  int slices;                   // S
  int a_row0, b_row0;           // first slice rows of the A and B sides
  const int* expo;              // e_r of every slice row (power-of-two row scales)
  int tiles_m, tiles_n;
  int* err;
};

// Instruction descriptor, kind::i8: INT32 accumulator (bits 4-5 = 2), A and B signed
// 8-bit (bits 7-9 = 1, 10-12 = 1), K-major, N >> 3 at 17-22, M >> 4 at 24-28.
__host__ __device__ constexpr uint32_t idesc_i8() {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem), "l"(adesc), "l"(bdesc), "r"(idesc_i8()), "r"(accumulate)
      : "memory");
}

// 2^e as a double, built from its exponent bits (normal range; 0 below it).
__device__ __forceinline__ double pow2(int e) {
  return e < -1022 ? 0.0 : __longlong_as_double((long long)(e + 1023) << 52);
}
// Exact int32 -> double on the FP64 pipe: (2^52 + 2^31 + x) - (2^52 + 2^31).
__device__ __forceinline__ double i32_to_f64(uint32_t bits) {
  return __hiloint2double(0x43300000, (int)(bits ^ 0x80000000u)) - 4503601774854144.0;
}

// Lower tiles (ti * BM + BM - 1 >= tj * BN) of an m x n region, row by row.
__device__ __forceinline__ bool tile_of(int t, const Params& p, int& ti, int& tj) {
  // tiles of tile-row ti: columns 0 .. min(tiles_n, (ti * BM + BM - 1) / BN + 1) - 1
  int acc = 0;
  for (int r = 0; r < p.tiles_m; ++r) {
    const int w = min(p.tiles_n, (r * BM + BM - 1) / BN + 1);
    if (t < acc + w) {
      ti = r;
      tj = t - acc;
      return true;
    }
    acc += w;
  }
  return false;
}

// Slices: one 2D k-major int8 tensor of S * R rows (slice t of slice row r at row
// t * R + r, row pitch kp bytes), seen through two maps with 128-row (A side, rows
// a_row0 + ..) and 64-row (B side, rows b_row0 + ..) boxes of 128 bytes.
__global__ void __launch_bounds__(THREADS, 1)
    update_kernel(const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb, Params p, int R,
                  const int* stop) {
  using namespace cuchol::tc;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t afull[A_STAGES], aempty[A_STAGES], bfull[B_STAGES], bempty[B_STAGES];
  __shared__ __align__(8) uint64_t accb[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int s_fail, s_mma_a, s_mma_b;
  __shared__ double s_pc[BN];   // 2^e of the tile's columns

  if (cta_aborted(stop)) return;
  int ti, tj;
  if (!tile_of(blockIdx.x, p, ti, tj)) return;
  const int row0 = ti * BM, col0 = tj * BN;
  uint8_t* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t* abuf = base;
  uint8_t* bbuf = base + A_STAGES * A_TILE;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int S = p.slices, nkh = (p.k + KMAX - 1) / KMAX;   // k halves of up to KMAX

  if (threadIdx.x == 0) {
    for (int s = 0; s < A_STAGES; ++s) { mbar_init(&afull[s], 1); mbar_init(&aempty[s], 1); }
    for (int s = 0; s < B_STAGES; ++s) { mbar_init(&bfull[s], 1); mbar_init(&bempty[s], 1); }
    mbar_init(&accb[0], 1);
    mbar_init(&accb[1], 1);
    s_fail = 0;
    s_mma_a = 0;
    s_mma_b = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < BN) {
    const int col = col0 + threadIdx.x;
    s_pc[threadIdx.x] = (col < p.n) ? pow2(p.expo[p.b_row0 + col]) : 0.0;
  }
  if (warp == 0) tmem_alloc(&tmem_slot, 512);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_slot;
  const int r = row0 + 32 * warp + lane;
  const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
  const double pr = (r < p.m) ? pow2(p.expo[p.a_row0 + r]) : 0.0;
  double* cp = p.c + (long long)r * p.crs;

  // the producer's and the MMA thread's positions in the rings carry over the passes
  int a_issued = 0, b_issued = 0, a_used = 0, b_used = 0;
  const int npass = (S + NACC - 1) / NACC;
  for (int pass = 0; pass < npass; ++pass) {
    const int dlo = pass * NACC, dhi = min(S - 1, dlo + NACC - 1);   // diagonals t + u (0-based)
    if (threadIdx.x == 0 && s_fail == 0) {
      bool ok = true;
      for (int kh = 0; kh < nkh && ok; ++kh) {
        const int kbox = (min(KMAX, p.k - kh * KMAX) + 127) / 128;
        const uint32_t a_bytes = (uint32_t)kbox * BM * 128, b_bytes = (uint32_t)kbox * BN * 128;
        for (int t = 0; t <= dhi && ok; ++t) {
          const int as = a_issued % A_STAGES;
          if (a_issued >= A_STAGES && !mbar_wait(&aempty[as], ((a_issued / A_STAGES) & 1) ^ 1)) { ok = false; break; }
          mbar_expect_tx(&afull[as], a_bytes);
          for (int kb = 0; kb < kbox; ++kb)
            tma_load_2d(&ma, &afull[as], abuf + as * A_TILE + kb * BM * 128, kh * KMAX + kb * 128,
                        t * R + p.a_row0 + row0);
          ++a_issued;
          for (int u = max(0, dlo - t); u <= dhi - t; ++u) {
            const int bs = b_issued % B_STAGES;
            if (b_issued >= B_STAGES && !mbar_wait(&bempty[bs], ((b_issued / B_STAGES) & 1) ^ 1)) {
              ok = false;
              break;
            }
            mbar_expect_tx(&bfull[bs], b_bytes);
            for (int kb = 0; kb < kbox; ++kb)
              tma_load_2d(&mb, &bfull[bs], bbuf + bs * B_TILE + kb * BN * 128, kh * KMAX + kb * 128,
                          u * R + p.b_row0 + col0);
            ++b_issued;
          }
        }
      }
      if (!ok) s_fail = 1;
    } else if (threadIdx.x == 32 && s_fail == 0) {
      bool ok = true;
      uint32_t inited = 0;   // accumulators written in this pass (the first MMA overwrites)
      fence_after();
      for (int kh = 0; kh < nkh && ok; ++kh) {
        const int kbox = (min(KMAX, p.k - kh * KMAX) + 127) / 128;
        for (int t = 0; t <= dhi && ok; ++t) {
          const int as = a_used % A_STAGES;
          if (!mbar_wait(&afull[as], (a_used / A_STAGES) & 1)) { ok = false; break; }
          ++a_used;
          fence_after();
          const uint32_t a0 = smem_u32(abuf + as * A_TILE);
          for (int u = max(0, dlo - t); u <= dhi - t; ++u) {
            const int bs = b_used % B_STAGES;
            if (!mbar_wait(&bfull[bs], (b_used / B_STAGES) & 1)) { ok = false; break; }
            ++b_used;
            fence_after();
            const uint32_t b0 = smem_u32(bbuf + bs * B_TILE);
            const int ai = t + u - dlo;
            const uint32_t acc = tmem + (uint32_t)(ai * BN);
            for (int kb = 0; kb < kbox; ++kb)
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                const uint32_t accumulate = ((inited >> ai) & 1u) | (uint32_t)(kb > 0 || kk > 0);
                mma_i8(acc, smem_desc(a0 + kb * BM * 128 + 32 * kk), smem_desc(b0 + kb * BN * 128 + 32 * kk),
                       accumulate);
              }
            inited |= 1u << ai;
            mma_commit(&bempty[bs]);
          }
          mma_commit(&aempty[as]);
        }
      }
      s_mma_a = a_used;
      s_mma_b = b_used;
      if (!ok) s_fail = 1;
      mma_commit(&accb[pass]);
    }
    __syncthreads();
    const bool acc_ok = mbar_wait(&accb[pass], 0);
    fence_after();
    if (!acc_ok) s_fail = 1;
    __syncthreads();
    if (s_fail != 0) break;
    // fold this pass's accumulators into C
#pragma unroll 1
    for (int h = 0; h < BN / 32; ++h) {
      double cv[32], accd[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) {      // C first: its loads overlap the TMEM reads
        const int col = col0 + 32 * h + i;
        cv[i] = (r < p.m && col < p.n && r >= col) ? cp[(long long)col * p.ccs] : 0.0;
        accd[i] = 0.0;
      }
#pragma unroll 1
      for (int d = dlo; d <= dhi; ++d) {
        const double sc = pow2(-7 * (d + 2));
        float v[32];
        tmem_ld32(trow + (d - dlo) * BN + 32 * h, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) accd[i] = fma(i32_to_f64(__float_as_uint(v[i])), sc, accd[i]);
      }
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int col = col0 + 32 * h + i;
        if (r < p.m && col < p.n && r >= col) cp[(long long)col * p.ccs] = cv[i] - accd[i] * pr * s_pc[32 * h + i];
      }
    }
    fence_before();   // the accumulators are read: the next pass may overwrite them
    __syncthreads();
  }
  if (s_fail != 0) {
    __syncthreads();
    if (threadIdx.x == 0) {
      // a wait gave up: let the loads still in flight land before the CTA exits
      for (int t = s_mma_a; t < a_issued; ++t) mbar_wait(&afull[t % A_STAGES], (t / A_STAGES) & 1);
      for (int b = s_mma_b; b < b_issued; ++b) mbar_wait(&bfull[b % B_STAGES], (b / B_STAGES) & 1);
      atomicExch(p.err, 1);
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// Slices of the rows of a panel P (logical P(r, l) = P[r * prs + l * pcs], rows
// [0, R), k columns): expo[r] = frexp exponent of max_l |P(r, l)|, and slice t of row r
// (t < S) at sl + (t * R + r) * kp, bytes l < k (the rest of the row pitch zero).
// CTA: 32 rows (lane = row), 8 warps over 16-column segments.
__global__ void __launch_bounds__(256)
    slice_kernel(const double* __restrict__ P, long long prs, long long pcs, int R, int k, int S, int8_t* sl,
                 long long kp, int* __restrict__ expo, const int* stop) {
  __shared__ int s_e[8][32];
  if (cta_aborted(stop)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r = blockIdx.x * 32 + lane;
  const int nseg = (int)(kp / 16);
  // row maximum
  double mx = 0.0;
  for (int sgi = warp; sgi < nseg; sgi += 8)
    for (int i = 0; i < 16; ++i) {
      const int l = sgi * 16 + i;
      if (r < R && l < k) mx = fmax(mx, fabs(P[(long long)r * prs + (long long)l * pcs]));
    }
  int e = 0;
  frexp(mx, &e);
  s_e[warp][lane] = e;
  __syncthreads();
  int er = s_e[0][lane];
  for (int w = 1; w < 8; ++w) er = max(er, s_e[w][lane]);
  if (warp == 0 && r < R) expo[r] = er;
  if (r >= R) return;
  for (int sgi = warp; sgi < nseg; sgi += 8) {
    double x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int l = sgi * 16 + i;
      x[i] = (l < k) ? ldexp(P[(long long)r * prs + (long long)l * pcs], -er) : 0.0;   // |x| < 1
    }
    for (int t = 0; t < S; ++t) {
      uint32_t w4[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        uint32_t wv = 0;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const double y = x[4 * q + b] * 128.0;      // exact
          const double a = trunc(y);                  // |a| <= 127
          x[4 * q + b] = y - a;                       // exact
          wv |= ((uint32_t)(uint8_t)(int8_t)(int)a) << (8 * b);
        }
        w4[q] = wv;
      }
      *reinterpret_cast<uint4*>(sl + ((long long)t * R + r) * kp + sgi * 16) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
  }
}

}  // namespace oz
}  // namespace cuchol
