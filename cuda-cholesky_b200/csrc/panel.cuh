// Diagonal-block kernels of the blocked factor and inverse (one CTA per block).
//
//   diag_factor_kernel  Cholesky factor L of one jb x jb diagonal block (jb <= 128),
//                       written back to A, plus (optionally) W = inv(L) with explicit
//                       zeros above the diagonal, which turns the panel solve
//                       L21 = A21 L11^-H into a plain tensor-core GEMM.  Also reports
//                       the first failing pivot and adds the block's log det share.
//   diag_invert_kernel  in-place inverse of every nb x nb diagonal block of a
//                       triangular matrix (the leaves of the recursive ?TRTRI).
//
// Both work on the block in shared memory in 32-column sub-blocks:
//   * the factor takes the block one 32-column sub-panel (the sub-block column from
//     its diagonal down) at a time: a left-looking register-tiled update by the
//     columns before it, then a right-looking factor of the sub-panel by all 256
//     threads, each holding 16 elements of one row in registers, one pivot per
//     step and one barrier per step (the next pivot column is published to shared
//     memory by the update that finishes it);
//   * the inverse (when asked for) inverts each 32 x 32 diagonal sub-block with one
//     warp (one column per lane) and assembles inv(L) block column by block column
//     from the last one back (the order of the reference's lower dtrtri,
//     lapack/dtrtri.c:141-162) with register-tiled SIMT products.
// The diagonal block is factored on the GPU next to the trailing update; the
// reference copied it to the host for a CPU dpotrf every step
// (lapack/dpotrf.c:263-276).
#pragma once
#include "scalar.cuh"

namespace cuchol {

// Asynchronous global -> shared copy of one element (cp.async: no register
// staging, every copy of a loop is in flight at once); valid = false writes zeros.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src, bool valid) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  const int n = valid ? (int)sizeof(T) : 0;
  if constexpr (sizeof(T) == 16) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(d), "l"(src), "n"(sizeof(T)), "r"(n)
                 : "memory");
  }
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

template <typename T>
__device__ __forceinline__ T shfl(T v, int src) {
  if constexpr (Traits<T>::complex) {
    v.x = __shfl_sync(0xffffffffu, v.x, src);
    v.y = __shfl_sync(0xffffffffu, v.y, src);
    return v;
  } else {
    return __shfl_sync(0xffffffffu, v, src);
  }
}

__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }

// Shared-memory layout of one block: column-major, leading dimension LD = NB + 1.
template <typename T, int NB>
struct DiagSmem {
  static constexpr int LD = NB + 1;
  static constexpr int NP = (NB + 31) / 32;          // 32-column sub-blocks
  static constexpr size_t S = sizeof(T) * NB * LD;    // the block
  static constexpr size_t X = sizeof(T) * NP * 32 * 33;   // inverted sub-blocks
  static constexpr int TLD = NB / 2 + 1;               // TMP: (NB/2) x (NB/2), row-major
  static constexpr size_t TMP = sizeof(T) * (NB / 2) * TLD;
  static constexpr size_t R = sizeof(T) * NB;         // reciprocal pivots
  static constexpr size_t C = sizeof(T) * 2 * 128;    // pivot columns (double-buffered)
  static constexpr size_t bytes = S + X + TMP + R + C + 16;
};

__device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_(double x) { return rsqrt(x); }

// 16 consecutive shared-memory elements from a 16-byte aligned address, in
// 16-byte loads.
template <typename T>
__device__ __forceinline__ void load16(const T* p, T (&v)[16]) {
  static_assert(16 % sizeof(T) == 0, "element of 4, 8 or 16 bytes");
  constexpr int per = 16 / sizeof(T);
  const int4* q = reinterpret_cast<const int4*>(p);
#pragma unroll
  for (int u = 0; u < 16 / per; ++u) {
    const int4 w = q[u];
    memcpy(&v[u * per], &w, 16);
  }
}

// Right-looking Cholesky of the sub-panel S(c0:jb, c0:c0+pb) (pb <= 32, jb - c0 <=
// 128), lower part, in place, by all 256 threads of the block (every thread must
// call it).  Thread t holds row c0 + (t & 127), columns c0 + 16 (t >> 7) + q
// (q = 0..15), in registers.  Step k:
//   d = A(k,k), r = 1/sqrt(d)             (every thread, from the published column)
//   L(i,k) = A(i,k) r                      (the owners of column k keep it)
//   A(i,j) -= (L(i,k) r) conj(A(j,k)), j > k
// and the owners of column k+1 publish it (rows k+1 ..) for the next step, so each
// step takes one barrier.  The steps of one 16-column half are unrolled (column k
// is register kq = k mod 16 of its owners, a compile-time index); the two halves
// are a loop.  Elements above the diagonal and rows past jb are computed on but
// never stored.  cbuf: 2 x 128 elements.  rdiag[c0+k] = 1/L(k,k).  Returns the
// first failing local column (pivot <= 0 or NaN) or -1, the same in every thread;
// on failure the columns before it are factored and the rest is left as updated.
// Ends with a barrier.
template <typename T, int NT>
__device__ __noinline__ int subpanel_chol(T* S, int LD, int c0, int pb, int jb, T* rdiag, T* cbuf) {
  static_assert(NT == 256, "one thread per (row, 16-column half) of a 128 x 32 sub-panel");
  using R = RealOf<T>;
  const int t = threadIdx.x;
  const int ii = t & 127;                 // local row
  const int h = t >> 7;                   // column half
  const bool row_ok = c0 + ii < jb;
  T x[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int j = 16 * h + q;
    x[q] = (row_ok && j < pb && ii >= j) ? S[(c0 + j) * LD + c0 + ii] : zero<T>();
  }
  if (h == 0 && row_ok) cbuf[ii] = x[0];
  __syncthreads();
  int fail = -1;
#pragma unroll 1
  for (int kk = 0; kk < 2 && 16 * kk < pb; ++kk) {
#pragma unroll
    for (int kq = 0; kq < 16; ++kq) {
      const int k = 16 * kk + kq;
      if (k >= pb) break;                 // the same in every thread
      const T* cur = cbuf + (k & 1) * 128;
      T* nxt = cbuf + ((k + 1) & 1) * 128;
      const R d = re(cur[k]);
      if (!(d > R(0))) {
        fail = k;
        break;
      }
      const R r = rsqrt_(d);
      const T li = (ii == k) ? from_real<T>(d * r) : scale(cur[ii], r);
      if (h == kk && ii >= k) x[kq] = li;
      if (t == 0) rdiag[c0 + k] = from_real<T>(r);
      const T lir = neg(scale(li, r));
      if (h == kk) {
        T v[16];
        load16(cur + 16 * kk, v);
#pragma unroll
        for (int q = kq + 1; q < 16; ++q) mac(x[q], lir, cj(v[q]));
      } else if (h > kk) {
        T v[16];
        load16(cur + 16, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) mac(x[q], lir, cj(v[q]));
      }
      if (k + 1 < pb && row_ok && ii >= k + 1) {
        if (kq < 15) {
          if (h == kk) nxt[ii] = x[kq + 1];
        } else if (h == kk + 1) {
          nxt[ii] = x[0];
        }
      }
      __syncthreads();
    }
    if (fail >= 0) break;
  }
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int j = 16 * h + q;
    if (row_ok && j < pb && ii >= j) S[(c0 + j) * LD + c0 + ii] = x[q];
  }
  __syncthreads();
  return fail;
}

// Warp: X = inv(L_pp) for the pb x pb lower sub-block at (c0, c0) (unit: implicit
// unit diagonal; rdiag[c0+i] = 1/L(i,i) otherwise).  Lane j computes column j in
// registers, unrolled:
//   X(j,j) = 1/L(j,j),  X(i,j) = -(1/L(i,i)) sum_{k=j..i-1} L(i,k) X(k,j).
// X(i, j) is stored at X[j*33 + i]: lower part written, upper part zero.
template <typename T>
__device__ __noinline__ void warp_inv32(const T* S, int LD, int c0, int pb, const T* rdiag, bool unit, T* X) {
  const int j = threadIdx.x & 31;
  T x[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const T ri = unit ? from_real<T>(RealOf<T>(1)) : (i < pb ? rdiag[c0 + i] : zero<T>());
    T s0 = zero<T>(), s1 = zero<T>();
#pragma unroll
    for (int k = 0; k < i; ++k) {
      if (k >= j) {
        const T l = S[(c0 + k) * LD + c0 + i];
        if (k & 1) mac(s1, l, x[k]); else mac(s0, l, x[k]);
      }
    }
    x[i] = (i < j || i >= pb || j >= pb) ? zero<T>() : (i == j ? ri : neg(mul(ri, add(s0, s1))));
  }
#pragma unroll
  for (int i = 0; i < 32; ++i) X[j * 33 + i] = x[i];
}

// S(r, c) -= sum_{k < c0} S(r, k) conj(S(c, k)) for rows [c0, nr), columns
// [c0, c0 + pb): 4 x 4 register tiles.
template <typename T, int NT>
__device__ void block_update(T* S, int LD, int c0, int pb, int nr) {
  const int ncq = 8;                                // column quads of the sub-block
  const int nrq = (nr - c0 + 3) / 4;                // row quads
  for (int t = threadIdx.x; t < nrq * ncq; t += NT) {
    const int r0 = c0 + 4 * (t / ncq), cb = c0 + 4 * (t % ncq);
    T acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = zero<T>();
#pragma unroll 4
    for (int k = 0; k < c0; ++k) {
      T a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = (r0 + u < nr) ? S[k * LD + r0 + u] : zero<T>();
#pragma unroll
      for (int v = 0; v < 4; ++v) b[v] = cj(S[k * LD + cb + v]);
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) mac(acc[u][v], a[u], b[v]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v)
        if (r0 + u < nr && cb + v < c0 + pb) S[(cb + v) * LD + r0 + u] = sub(S[(cb + v) * LD + r0 + u], acc[u][v]);
  }
}

// W(R, C) = -W(R, R) L(R, C) W(C, C) for the row block R = [r0, r0 + nr) and the
// column block C = [c0, c0 + nc) (r0 >= c0 + nc), where the diagonal blocks of S
// already hold the inverses W(R, R) and W(C, C) (lower parts; the upper parts of
// diagonal blocks are not read) and S(R, C) still holds L(R, C).  Two 4 x 4
// register-tiled products through TMP (row-major, ld tld).
template <typename T, int NT>
__device__ void inverse_offdiag(T* S, int LD, int r0, int nr, int c0, int nc, T* TMP, int tld) {
  // TMP(r, c) = sum_{k >= c} L(r0 + r, c0 + k) W(c0 + k, c0 + c)
  for (int t = threadIdx.x; t < ((nr + 3) / 4) * ((nc + 3) / 4); t += NT) {
    const int rb = 4 * (t % ((nr + 3) / 4)), cb = 4 * (t / ((nr + 3) / 4));
    T acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = zero<T>();
#pragma unroll 4
    for (int k = cb; k < nc; ++k) {
      T a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = (rb + u < nr) ? S[(c0 + k) * LD + r0 + rb + u] : zero<T>();
#pragma unroll
      for (int v = 0; v < 4; ++v) b[v] = (cb + v < nc && k >= cb + v) ? S[(c0 + cb + v) * LD + c0 + k] : zero<T>();
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) mac(acc[u][v], a[u], b[v]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v)
        if (rb + u < nr && cb + v < nc) TMP[(rb + u) * tld + cb + v] = acc[u][v];
  }
  __syncthreads();
  // S(r0 + r, c0 + c) = -sum_{k <= r} W(r0 + r, r0 + k) TMP(k, c)
  for (int t = threadIdx.x; t < ((nr + 3) / 4) * ((nc + 3) / 4); t += NT) {
    const int rb = 4 * (t % ((nr + 3) / 4)), cb = 4 * (t / ((nr + 3) / 4));
    T acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = zero<T>();
#pragma unroll 4
    for (int k = 0; k < min(nr, rb + 4); ++k) {
      T a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = (rb + u < nr && k <= rb + u) ? S[(r0 + k) * LD + r0 + rb + u] : zero<T>();
#pragma unroll
      for (int v = 0; v < 4; ++v) b[v] = (cb + v < nc) ? TMP[k * tld + cb + v] : zero<T>();
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) mac(acc[u][v], a[u], b[v]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v)
        if (rb + u < nr && cb + v < nc) S[(c0 + cb + v) * LD + r0 + rb + u] = neg(acc[u][v]);
  }
  __syncthreads();
}

// In-place inverse of the lower jb x jb block in S (jb <= 128), given the inverted
// 32 x 32 diagonal sub-blocks X[p] (X(i, j) of block p at X[p*32*33 + j*33 + i]):
// [L11 0; L21 L22]^-1 = [W11 0; -W22 L21 W11, W22], applied to pairs of 32-blocks
// and then to pairs of 64-blocks.
template <typename T, int NT>
__device__ void assemble_inverse(T* S, int LD, int jb, const T* X, T* TMP, int tld) {
  const int np = (jb + 31) / 32;
  for (int t = threadIdx.x; t < np * 32 * 32; t += NT) {
    const int p = t / 1024, e = t % 1024, i = e % 32, c = e / 32;
    if (32 * p + i < jb && 32 * p + c < jb && i >= c) S[(32 * p + c) * LD + 32 * p + i] = X[p * 32 * 33 + c * 33 + i];
  }
  __syncthreads();
  for (int b = 32; b < jb; b *= 2) {
    for (int c0 = 0; c0 + b < jb; c0 += 2 * b) {
      const int r0 = c0 + b;
      inverse_offdiag<T, NT>(S, LD, r0, min(b, jb - r0), c0, b, TMP, tld);
    }
  }
}

// Factor (and optionally invert) one jb x jb diagonal block, jb <= NB.
//   A     : top-left of the block in the logical lower view (strides rs, cs)
//   W     : if not null, inv(L) as a full jb x jb matrix (ldw), zeros above the diagonal
// On failure at local column k: *d_info = info_base + k + 1 (if still 0), the
// partially factored block is written back, W is not written.
template <typename T, int NB, int NT>
__device__ __forceinline__ void diag_factor_block(T* __restrict__ A, long long rs, long long cs, int jb,
                                                  T* __restrict__ W, int ldw, long long info_base,
                                                  int* __restrict__ d_info, double* __restrict__ logdet) {
  using R = RealOf<T>;
  using L = DiagSmem<T, NB>;
  constexpr int LD = L::LD;
  if (cta_aborted(d_info)) return;   // an earlier block already failed
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S = reinterpret_cast<T*>(smem_raw);
  T* X = reinterpret_cast<T*>(smem_raw + L::S);
  T* TMP = reinterpret_cast<T*>(smem_raw + L::S + L::X);
  T* rdiag = reinterpret_cast<T*>(smem_raw + L::S + L::X + L::TMP);
  T* cbuf = reinterpret_cast<T*>(smem_raw + L::S + L::X + L::TMP + L::R);
  __shared__ int s_fail;
  const int tid = threadIdx.x;
  const bool rows_fast = (rs == 1);

  for (int e = tid; e < jb * jb; e += NT) {
    int r, c;
    if (rows_fast) { r = e % jb; c = e / jb; } else { c = e % jb; r = e / jb; }
    cp_async_elem<T>(&S[c * LD + r], r >= c ? A + r * rs + c * cs : A, r >= c);
  }
  if (tid == 0) s_fail = -1;
  cp_async_wait_all();
  __syncthreads();

  const int np = (jb + 31) / 32;
  for (int p = 0; p < np; ++p) {
    const int c0 = 32 * p, pb = min(32, jb - c0);
    if (p > 0) {
      block_update<T, NT>(S, LD, c0, pb, jb);
      __syncthreads();
    }
    const int f = subpanel_chol<T, NT>(S, LD, c0, pb, jb, rdiag, cbuf);
    if (f >= 0) {
      if (tid == 0) s_fail = c0 + f;
      __syncthreads();
      break;
    }
  }

  // the factor (lower part) back to A
  for (int e = tid; e < jb * jb; e += NT) {
    int r, c;
    if (rows_fast) { r = e % jb; c = e / jb; } else { c = e % jb; r = e / jb; }
    if (r >= c) A[r * rs + c * cs] = S[c * LD + r];
  }
  if (s_fail >= 0) {
    if (tid == 0) atomicCAS(d_info, 0, (int)(info_base + s_fail + 1));
    return;
  }
  if (logdet != nullptr) {
    // 2 sum log L(j,j), reduced by warp 0 in a fixed order (deterministic)
    if (tid < 32) {
      double s = 0.0;
      for (int jj = tid; jj < jb; jj += 32) s += log((double)re(S[jj * LD + jj]));
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (tid == 0) *logdet += 2.0 * s;
    }
  }
  if (W == nullptr) return;
  __syncthreads();
  for (int p = tid / 32; p < np; p += NT / 32)
    warp_inv32<T>(S, LD, 32 * p, min(32, jb - 32 * p), rdiag, false, X + p * 32 * 33);
  __syncthreads();
  assemble_inverse<T, NT>(S, LD, jb, X, TMP, L::TLD);
  for (int e = tid; e < jb * jb; e += NT) {
    const int r = e % jb, c = e / jb;
    W[r + (long long)c * ldw] = (r >= c) ? S[c * LD + r] : zero<T>();
  }
}

// In-place inverse of the diagonal blocks [b*nb, b*nb + jb) of a triangular matrix
// (blockIdx.x = b), nb <= NB.  Only the lower triangle of each block is read or
// written; unit: the diagonal is taken as 1 and left untouched.
template <typename T, int NB, int NT>
__global__ void __launch_bounds__(NT)
diag_factor_kernel(T* __restrict__ A, long long rs, long long cs, int jb, T* __restrict__ W, int ldw,
                   long long info_base, int* __restrict__ d_info, double* __restrict__ logdet) {
  diag_factor_block<T, NB, NT>(A, rs, cs, jb, W, ldw, info_base, d_info, logdet);
}

// One diagonal block of one matrix of a batch (batched factor: one CTA per task).
template <typename T>
struct DiagTask {
  T* a;               // top-left of the block, logical lower view (strides rs, cs)
  long long rs, cs;
  int jb;
  T* w;               // inverse of the factored block (ld ldw), or null
  int ldw;
  long long info_base;
  int* info;          // the matrix's info word (later steps skip once it is set)
  double* logdet;     // the matrix's log det accumulator, or null
};

template <typename T, int NB, int NT>
__global__ void __launch_bounds__(NT) diag_factor_batched_kernel(const DiagTask<T>* __restrict__ tasks) {
  const DiagTask<T> t = tasks[blockIdx.x];
  diag_factor_block<T, NB, NT>(t.a, t.rs, t.cs, t.jb, t.w, t.ldw, t.info_base, t.info, t.logdet);
}

template <typename T, int NB, int NT>
__device__ __forceinline__ void diag_invert_block(T* __restrict__ B, long long rs, long long cs, int jb,
                                                  int unit);

template <typename T, int NB, int NT>
__global__ void __launch_bounds__(NT)
diag_invert_kernel(T* __restrict__ A, long long rs, long long cs, int n, int nb, int unit) {
  const int o = blockIdx.x * nb;
  diag_invert_block<T, NB, NT>(A + o * rs + o * cs, rs, cs, min(nb, n - o), unit);
}

// In-place inverse of one diagonal block of one matrix of a batch.
template <typename T>
struct InvTask {
  T* b;               // top-left of the block (strides rs, cs)
  long long rs, cs;
  int jb;
  int unit;
  const int* stop;    // skip when this word is non-zero (the matrix's factor failed)
};

template <typename T, int NB, int NT>
__global__ void __launch_bounds__(NT) diag_invert_batched_kernel(const InvTask<T>* __restrict__ tasks) {
  const InvTask<T> t = tasks[blockIdx.x];
  if (cta_aborted(t.stop)) return;
  diag_invert_block<T, NB, NT>(t.b, t.rs, t.cs, t.jb, t.unit);
}

template <typename T, int NB, int NT>
__device__ __forceinline__ void diag_invert_block(T* __restrict__ B, long long rs, long long cs, int jb,
                                                  int unit) {
  using R = RealOf<T>;
  using L = DiagSmem<T, NB>;
  constexpr int LD = L::LD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S = reinterpret_cast<T*>(smem_raw);
  T* X = reinterpret_cast<T*>(smem_raw + L::S);
  T* TMP = reinterpret_cast<T*>(smem_raw + L::S + L::X);
  T* rdiag = reinterpret_cast<T*>(smem_raw + L::S + L::X + L::TMP);
  const bool rows_fast = (rs == 1);
  for (int e = threadIdx.x; e < jb * jb; e += NT) {
    int r, c;
    if (rows_fast) { r = e % jb; c = e / jb; } else { c = e % jb; r = e / jb; }
    cp_async_elem<T>(&S[c * LD + r], r >= c ? B + r * rs + c * cs : B, r >= c);
  }
  cp_async_wait_all();
  __syncthreads();
  for (int i = threadIdx.x; i < jb; i += NT) rdiag[i] = unit ? from_real<T>(R(1)) : recip(S[i * LD + i]);
  __syncthreads();
  const int np = (jb + 31) / 32;
  const int w = threadIdx.x / 32;
  for (int p = w; p < np; p += NT / 32)
    warp_inv32<T>(S, LD, 32 * p, min(32, jb - 32 * p), rdiag, unit != 0, X + p * 32 * 33);
  __syncthreads();
  assemble_inverse<T, NT>(S, LD, jb, X, TMP, L::TLD);
  for (int e = threadIdx.x; e < jb * jb; e += NT) {
    int r, c;
    if (rows_fast) { r = e % jb; c = e / jb; } else { c = e % jb; r = e / jb; }
    if (r > c || (r == c && !unit)) B[r * rs + c * cs] = S[c * LD + r];
  }
}

}  // namespace cuchol
