// Tile engine: every BLAS3 step of the path is one or more "problems"
//
//     C(i, j) = alpha * sum_k opA(Ahat(i, k)) * opB(Bhat(j, k)) + beta * Cin(i, j)
//
// over i < m, j < n, where Ahat / Bhat are strided views (row stride, k stride),
// op is the identity or complex conjugation, and either view may be triangular
// (its entries outside the triangle are treated as zero and never read, because
// they belong to the other triangle of the caller's matrix).  This covers the
// path's SYRK/HERK (trailing update), GEMM (lookahead update), TRSM (as a product
// with the inverted diagonal block) and TRMM (TRTRI / LAUUM) steps.
//
// A launch takes one problem by value, or a list of problems in device memory
// (a grouped launch: all nodes of one level of the recursive TRTRI, for example).
#pragma once
#include <stdint.h>
#include "scalar.cuh"

namespace cuchol {

enum : uint8_t { TRI_NONE = 0, TRI_LOWER = 1 /* nonzero iff k <= row */, TRI_UPPER = 2 /* nonzero iff k >= row */ };

template <typename T>
struct GemmProblem {
  const T* a; long long a_rs, a_ks;   // Ahat(i, k) = a[i*a_rs + k*a_ks]
  const T* b; long long b_rs, b_ks;   // Bhat(j, k) = b[j*b_rs + k*b_ks]
  T* c; long long c_rs, c_cs;         // C(i, j)    = c[i*c_rs + j*c_cs]
  const T* cin; long long cin_rs, cin_cs;
  int m, n, k;
  T alpha, beta;
  uint8_t conj_a, conj_b, tri_a, tri_b;
  uint8_t unit_a, unit_b;   // a triangular view has an implicit unit diagonal
  uint8_t lower_only;   // write only i >= j; tiles wholly above the diagonal exit
  uint8_t real_diag;    // store Im C(i, i) = 0 (Hermitian results)
  const int* stop;      // grouped launches: skip the problem when this word is set
  int tiles_n;          // tile columns of this problem (filled by the launcher)
  int tile_begin;       // first tile index of this problem in a grouped launch
};

template <typename T>
struct GemmLaunch {
  GemmProblem<T> single;          // used when list == nullptr
  const GemmProblem<T>* list;     // grouped launch: problems sorted by tile_begin
  int nlist;
};

template <typename T>
__device__ __forceinline__ const GemmProblem<T>* find_problem(const GemmLaunch<T>& L, int tile) {
  if (L.list == nullptr) return &L.single;
  int lo = 0, hi = L.nlist - 1;
  while (lo < hi) {   // last problem with tile_begin <= tile
    int mid = (lo + hi + 1) >> 1;
    if (L.list[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
  }
  return &L.list[lo];
}

// k range of a tile whose rows are [i0, i0+BM) and columns [j0, j0+BN)
template <typename T>
__device__ __forceinline__ void tile_k_range(const GemmProblem<T>& P, int i0, int j0, int BM, int BN,
                                             int& kb, int& ke) {
  kb = 0; ke = P.k;
  if (P.tri_a == TRI_LOWER) ke = min(ke, i0 + BM);
  if (P.tri_a == TRI_UPPER) kb = max(kb, i0);
  if (P.tri_b == TRI_LOWER) ke = min(ke, j0 + BN);
  if (P.tri_b == TRI_UPPER) kb = max(kb, j0);
}

__device__ __forceinline__ bool tri_keep(uint8_t tri, int row, int k) {
  return tri == TRI_NONE || (tri == TRI_LOWER ? k <= row : k >= row);
}

// ---------------------------------------------------------------------------------
// SIMT engine (all four types): 64 x 64 tiles, 256 threads, 4 x 4 outputs each,
// double-buffered shared memory with register prefetch.  LA / LB select which index
// of each view is contiguous in memory (0: rows, 1: k) so global loads coalesce.
// ---------------------------------------------------------------------------------
template <typename T> struct SimtCfg { static constexpr int BK = 16; };
template <> struct SimtCfg<cuDoubleComplex> { static constexpr int BK = 8; };

// TM x TM outputs per thread (strided by 16), a 16TM x 16TM tile per CTA: TM = 4 for
// every type in grouped launches; TM = 8 (128 x 128 tiles, 64 FMAs per 16 shared
// loads) for large single FP32 products with a long k, where the 4 x 4 tile is bound by
// shared-memory loads.
template <typename T, int LA, int LB, int TM = 4>
__global__ void __launch_bounds__(256)
gemm_simt_kernel(const __grid_constant__ GemmLaunch<T> L, const int* __restrict__ abort_flag) {
  constexpr int BM = 16 * TM, BN = 16 * TM, BK = SimtCfg<T>::BK, NT = 256;
  constexpr int LDA_PER = BM * BK / NT, LDB_PER = BN * BK / NT;
  const GemmProblem<T>& P = *find_problem(L, blockIdx.x);
  if (cta_aborted(abort_flag, P.stop)) return;
  const int tile = blockIdx.x - P.tile_begin;
  const int ti = tile / P.tiles_n, tj = tile % P.tiles_n;
  const int i0 = ti * BM, j0 = tj * BN;
  if (P.lower_only && j0 > i0 + BM - 1) return;
  int kb, ke;
  tile_k_range(P, i0, j0, BM, BN, kb, ke);

  __shared__ T As[2][BK][BM + 1];
  __shared__ T Bs[2][BK][BN + 1];
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;

  T acc[TM][TM];
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TM; ++b) acc[a][b] = zero<T>();

  T ra[LDA_PER], rb[LDB_PER];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < LDA_PER; ++q) {
      const int e = tid + q * NT;
      const int r = (LA == 0) ? e % BM : e / BK;
      const int kk = (LA == 0) ? e / BM : e % BK;
      const int i = i0 + r, k = k0 + kk;
      T v = zero<T>();
      if (i < P.m && k < ke && k >= kb && tri_keep(P.tri_a, i, k))
        v = (P.unit_a && i == k) ? from_real<T>(RealOf<T>(1)) : P.a[i * P.a_rs + k * P.a_ks];
      ra[q] = P.conj_a ? cj(v) : v;
    }
#pragma unroll
    for (int q = 0; q < LDB_PER; ++q) {
      const int e = tid + q * NT;
      const int r = (LB == 0) ? e % BN : e / BK;
      const int kk = (LB == 0) ? e / BN : e % BK;
      const int j = j0 + r, k = k0 + kk;
      T v = zero<T>();
      if (j < P.n && k < ke && k >= kb && tri_keep(P.tri_b, j, k))
        v = (P.unit_b && j == k) ? from_real<T>(RealOf<T>(1)) : P.b[j * P.b_rs + k * P.b_ks];
      rb[q] = P.conj_b ? cj(v) : v;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int q = 0; q < LDA_PER; ++q) {
      const int e = tid + q * NT;
      const int r = (LA == 0) ? e % BM : e / BK;
      const int kk = (LA == 0) ? e / BM : e % BK;
      As[buf][kk][r] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < LDB_PER; ++q) {
      const int e = tid + q * NT;
      const int r = (LB == 0) ? e % BN : e / BK;
      const int kk = (LB == 0) ? e / BN : e % BK;
      Bs[buf][kk][r] = rb[q];
    }
  };

  // align the first k block down to BK so that tiles of one problem share blocks
  int k0 = (kb / BK) * BK;
  if (k0 < ke) {
    load(k0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (; k0 < ke; k0 += BK) {
      const bool more = (k0 + BK < ke);
      if (more) load(k0 + BK);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        T av[TM], bv[TM];
#pragma unroll
        for (int a = 0; a < TM; ++a) av[a] = As[buf][kk][tx + 16 * a];
#pragma unroll
        for (int b = 0; b < TM; ++b) bv[b] = Bs[buf][kk][ty + 16 * b];
#pragma unroll
        for (int a = 0; a < TM; ++a)
#pragma unroll
          for (int b = 0; b < TM; ++b) mac(acc[a][b], av[a], bv[b]);
      }
      if (more) {
        store(buf ^ 1);
        __syncthreads();
        buf ^= 1;
      }
    }
  }

#pragma unroll
  for (int a = 0; a < TM; ++a) {
    const int i = i0 + tx + 16 * a;
#pragma unroll
    for (int b = 0; b < TM; ++b) {
      const int j = j0 + ty + 16 * b;
      if (i < P.m && j < P.n && (!P.lower_only || i >= j)) {
        T v = mul(P.alpha, acc[a][b]);
        if (P.cin != nullptr) v = add(v, mul(P.beta, P.cin[i * P.cin_rs + j * P.cin_cs]));
        if constexpr (Traits<T>::complex) {
          if (P.real_diag && i == j) v.y = 0;
        }
        P.c[i * P.c_rs + j * P.c_cs] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------------
// FP64 tensor-core form of the grouped engine: the same problems, tiles (64 x 64,
// numbered as by gemm_simt_kernel) and masked, coalesced global loads (register
// staged, double-buffered shared memory), with the products on the warp-level DMMA
// instruction (mma.sync m16n8k4 f64): four warps of 32 x 32 outputs (2 m16 x 4 n8
// blocks).  Shared rows hold one k of 64 rows, padded to 68 doubles, so that the
// 16 lanes of each half warp (rows g = 0..3 or 4..7, k slots t = 0..3) read 16
// distinct bank pairs: 2g + 8t mod 32.  Used for FP64 problems that the TMA-fed
// engine does not take: grouped launches (problem lists of many small products,
// the batched plans and the recursive ?trtri levels) and unaligned views.
// ---------------------------------------------------------------------------------
constexpr int kDgBM = 64, kDgBK = 16, kDgThreads = 128, kDgLD = kDgBM + 4;

__device__ __forceinline__ void dmma_m16n8k4(double (&d)[4], double a0, double a1, double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b));
}

template <int LA, int LB>
__global__ void __launch_bounds__(kDgThreads)
gemm_dmma_group_kernel(const __grid_constant__ GemmLaunch<double> L, const int* __restrict__ abort_flag) {
  constexpr int BM = kDgBM, BN = kDgBM, BK = kDgBK, NT = kDgThreads, LDS = kDgLD;
  constexpr int PER = BM * BK / NT;   // elements of each operand a thread loads per k block
  const GemmProblem<double>& P = *find_problem(L, blockIdx.x);
  if (cta_aborted(abort_flag, P.stop)) return;
  const int tile = blockIdx.x - P.tile_begin;
  const int ti = tile / P.tiles_n, tj = tile % P.tiles_n;
  const int i0 = ti * BM, j0 = tj * BN;
  if (P.lower_only && j0 > i0 + BM - 1) return;
  int kb, ke;
  tile_k_range(P, i0, j0, BM, BN, kb, ke);

  __shared__ __align__(16) double As[2][BK][LDS];
  __shared__ __align__(16) double Bs[2][BK][LDS];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp & 1, wn = warp >> 1;   // warp rows wm*32 .., columns wn*32 ..
  double acc[2][4][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;

  double ra[PER], rb[PER];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = tid + q * NT;
      const int r = (LA == 0) ? e % BM : e / BK;
      const int kk = (LA == 0) ? e / BM : e % BK;
      const int i = i0 + r, k = k0 + kk;
      double v = 0.0;
      if (i < P.m && k < ke && k >= kb && tri_keep(P.tri_a, i, k)) v = (P.unit_a && i == k) ? 1.0 : P.a[i * P.a_rs + k * P.a_ks];
      ra[q] = v;
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = tid + q * NT;
      const int r = (LB == 0) ? e % BN : e / BK;
      const int kk = (LB == 0) ? e / BN : e % BK;
      const int j = j0 + r, k = k0 + kk;
      double v = 0.0;
      if (j < P.n && k < ke && k >= kb && tri_keep(P.tri_b, j, k)) v = (P.unit_b && j == k) ? 1.0 : P.b[j * P.b_rs + k * P.b_ks];
      rb[q] = v;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = tid + q * NT;
      const int r = (LA == 0) ? e % BM : e / BK;
      const int kk = (LA == 0) ? e / BM : e % BK;
      As[buf][kk][r] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = tid + q * NT;
      const int r = (LB == 0) ? e % BN : e / BK;
      const int kk = (LB == 0) ? e / BN : e % BK;
      Bs[buf][kk][r] = rb[q];
    }
  };

  int k0 = (kb / BK) * BK;
  if (k0 < ke) {
    load(k0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (; k0 < ke; k0 += BK) {
      const bool more = (k0 + BK < ke);
      if (more) load(k0 + BK);
#pragma unroll
      for (int k4 = 0; k4 < BK; k4 += 4) {
        const int kk = k4 + t;
        double a0[2], a1[2], bv[4];
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
          a0[mb] = As[buf][kk][wm * 32 + mb * 16 + g];
          a1[mb] = As[buf][kk][wm * 32 + mb * 16 + g + 8];
        }
#pragma unroll
        for (int nb8 = 0; nb8 < 4; ++nb8) bv[nb8] = Bs[buf][kk][wn * 32 + nb8 * 8 + g];
#pragma unroll
        for (int mb = 0; mb < 2; ++mb)
#pragma unroll
          for (int nb8 = 0; nb8 < 4; ++nb8) dmma_m16n8k4(acc[mb][nb8], a0[mb], a1[mb], bv[nb8]);
      }
      if (more) {
        store(buf ^ 1);
        __syncthreads();
        buf ^= 1;
      }
    }
  }

#pragma unroll
  for (int mb = 0; mb < 2; ++mb)
#pragma unroll
    for (int nb8 = 0; nb8 < 4; ++nb8)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int i = i0 + wm * 32 + mb * 16 + g + (e >> 1) * 8;
        const int j = j0 + wn * 32 + nb8 * 8 + 2 * t + (e & 1);
        if (i < P.m && j < P.n && (!P.lower_only || i >= j)) {
          double v = P.alpha * acc[mb][nb8][e];
          if (P.cin != nullptr) v = fma(P.beta, P.cin[i * P.cin_rs + j * P.cin_cs], v);
          P.c[i * P.c_rs + j * P.c_cs] = v;
        }
      }
}

}  // namespace cuchol
