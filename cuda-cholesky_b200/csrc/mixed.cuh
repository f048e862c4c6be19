// Mixed-precision SPD solve and the FP64 triangular solves under it (included at
// the end of lapack.cu; uses its launch helpers).  No counterpart in the reference
// library, which stops at ?potrf / ?potri (lapack/dpotrf.c:172, lapack/dpotri.c:25):
// the solve follows LAPACK's DSPOSV contract (low-precision factor, FP64
// refinement, FP64 fallback) on the dense SPD path of this library.
//
// Factor (cuDcholMixedCreate):
//   1. s_i = 1 / sqrt(a_ii); W = S A S + shift * I in FP32 (lower, our own buffer):
//      the symmetric diagonal scaling removes the row/column scaling part of
//      kappa(A) before any rounding to low precision.  The shift starts at u / 16 (u
//      the operand unit roundoff) and grows 8x after a breakdown.
//   2. Right-looking blocked Cholesky of W with the two-stream schedule of ?potrf
//      (outer blocks of 512 columns = four 128-column sub-panels, lookahead 1):
//        - diagonal blocks in FP64 (the ?potrf diagonal kernel on an FP64 copy),
//        - panel solve P = W21 inv(L11)^T in FP32 (SIMT engine) into a k-major
//          buffer, then copied into W and rounded to the operand type Q (BF16 or
//          TF32),
//        - trailing updates W22 -= Q Q^T on the tcgen05 tensor cores with FP32
//          accumulation (tc.cuh).
//   3. The inverses of W's 64 x 64 diagonal blocks (for the triangular solves).
// Solve (cuDcholMixedSolve): preconditioned conjugate gradients in FP64 on A x = b
// with M^-1 = S L^-T L^-1 S, in groups of 16 right-hand sides, as iterative
// refinement: the loop ends when every normwise backward error
//   |b - A x|_inf / (|A|_inf |x|_inf + |b|_inf)
// computed from a freshly formed FP64 residual is below the tolerance.
// A x uses the FP64 A in the caller's storage (symmetric product from one
// triangle, deterministic); the triangular solves are single launches in which
// row blocks are taken in ticket order and wait (bounded) for the blocks they
// depend on.

#include "tc.cuh"

namespace {
namespace mx {

constexpr int SB = 128;        // sub-panel width: FP64 diagonal blocks
constexpr int OB = 4 * SB;     // outer block: trailing updates with k = 512
constexpr int BS = 64;         // triangular-solve block
constexpr int NR = 16;         // right-hand sides per group
constexpr int SY = 256;        // symmetric-product tile
constexpr int NBT = 2048;      // preconditioner block (inverted diagonal blocks)
constexpr int kThreads = 256;

// ---- factor kernels --------------------------------------------------------------

// s_i = 1 / sqrt(A(i, i)); a diagonal that is not positive sets *bad.
__global__ void scale_kernel(const double* __restrict__ A, long long dstride, int n, double* __restrict__ s,
                             int* __restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = A[(long long)i * dstride];
  if (!(a > 0.0)) atomicExch(bad, 1);
  s[i] = (a > 0.0) ? 1.0 / sqrt(a) : 0.0;
}

// W(i, j) = s_i A(i, j) s_j (+ shift on the diagonal) for i >= j, FP32.  A is the
// logical lower view A(i, j) = a[i*rs + j*cs]; 32 x 32 tiles through shared memory
// so that both the read (either storage) and the write are coalesced.
__global__ void build_kernel(const double* __restrict__ a, long long rs, long long cs, int n,
                             const double* __restrict__ s, float shift, float* __restrict__ W, long long ldw) {
  __shared__ double t[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  if (j0 > i0 + 31) return;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
  const bool row_contig = (rs == 1);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int r = ty + 8 * k;
    // element (ii, jj) of the tile read by this thread
    const int ii = row_contig ? tx : r, jj = row_contig ? r : tx;
    const int i = i0 + ii, j = j0 + jj;
    t[ii][jj] = (i < n && j < n && i >= j) ? a[(long long)i * rs + (long long)j * cs] : 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int jj = ty + 8 * k, i = i0 + tx, j = j0 + jj;
    if (i < n && j < n && i >= j) {
      float w = (float)(s[i] * t[tx][jj] * s[j]);
      if (i == j) w += shift;
      W[i + (long long)j * ldw] = w;
    }
  }
}

// FP32 diagonal block of W -> FP64 copy D (ld SB); column j = blockIdx.x.
__global__ void diag_in_kernel(const float* __restrict__ W, long long ldw, int jb, double* __restrict__ D,
                               const int* __restrict__ stop) {
  if (cta_aborted(stop)) return;
  const int j = blockIdx.x, i = threadIdx.x;
  if (i < jb && i >= j) D[i + j * SB] = (double)W[i + (long long)j * ldw];
}

// Factored FP64 block -> W (FP32).
__global__ void diag_out_kernel(const double* __restrict__ D, int jb, float* __restrict__ W, long long ldw,
                                const int* __restrict__ stop) {
  if (cta_aborted(stop)) return;
  const int j = blockIdx.x, i = threadIdx.x;
  if (i < jb && i >= j) W[i + (long long)j * ldw] = (float)D[i + j * SB];
}

// ---- triangular solves ------------------------------------------------------------

// Inverse of the 64 x 64 diagonal blocks of a lower-triangular L (logical view
// L(i, j) = L[i*rs + j*cs]); DI[b] is column-major 64 x 64 with zeros above the
// diagonal.  Rows past n of the last block are given a unit diagonal.  One CTA per
// block, one thread per column of the inverse (forward substitution).
template <typename T>
__global__ void __launch_bounds__(BS) block_inverse_kernel(const T* __restrict__ L, long long rs, long long cs,
                                                           int n, T* __restrict__ DI) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls = reinterpret_cast<T*>(smem_raw);   // [BS][BS + 1], row-major
  T* X = Ls + BS * (BS + 1);                // [BS][BS + 1]
  const int b = blockIdx.x, i0 = b * BS, t = threadIdx.x;
  const bool row_contig = (rs == 1);
  for (int e = t; e < BS * BS; e += BS) {
    const int i = row_contig ? (e % BS) : (e / BS), j = row_contig ? (e / BS) : (e % BS);
    T v = T(0);
    if (i0 + i < n && i >= j) v = L[(long long)(i0 + i) * rs + (long long)(i0 + j) * cs];
    if (i0 + i >= n && i == j) v = T(1);
    Ls[i * (BS + 1) + j] = v;
  }
  __syncthreads();
  const int c = t;   // column of the inverse
  for (int i = 0; i < BS; ++i) {
    T x = T(0);
    if (i >= c) {
      T acc = (i == c) ? T(1) : T(0);
      for (int k = c; k < i; ++k) acc -= Ls[i * (BS + 1) + k] * X[k * (BS + 1) + c];
      x = acc / Ls[i * (BS + 1) + i];
    }
    X[i * (BS + 1) + c] = x;
  }
  __syncthreads();
  T* out = DI + (size_t)b * BS * BS;
  for (int e = t; e < BS * BS; e += BS) out[e] = X[(e % BS) * (BS + 1) + e / BS];
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0 waits until *ready >= need, for at most `limit` polls (limit < 0: 2^24,
// seconds); returns the value seen.  A wait that gives up sets *err and returns
// `need`, so that the solve still ends (with a wrong result the host then discards).
__device__ __forceinline__ unsigned wait_ready(const unsigned* ready, unsigned need, int* err, int limit) {
  const unsigned polls = limit < 0 ? (1u << 24) : (unsigned)limit;
  for (unsigned it = 0; it < polls; ++it) {
    const unsigned v = ld_acquire(ready);
    if (v >= need) return v;
    if (it > 64) __nanosleep(64);
  }
  atomicExch(err, 1);
  return need;
}

// Y := L^-1 (sc .* B) for up to NR right-hand sides; L lower (view strides rs, cs),
// B of type VB (ldb), Y of type T (ldy, at least 64 * ceil(n / 64) rows).  One CTA
// per 64-row block, blocks taken in ticket order; block I accumulates L(I, J) y_J
// for J < I as the y_J are published (the counter ready = number of finished
// blocks), then applies DI_I.
// Counters: ctr[0] ticket, ctr[1] ready; both zero at launch.
template <typename T, typename VB>
__global__ void __launch_bounds__(kThreads)
    trsv_fwd_kernel(const T* __restrict__ L, long long rs, long long cs, int n, const T* __restrict__ DI,
                    const VB* __restrict__ B, long long ldb, const double* __restrict__ sc, T* Y, long long ldy,
                    int nrhs, unsigned* ctr, int* err, int wait_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto Ls = reinterpret_cast<T(*)[BS + 1]>(smem_raw);           // [BS][BS + 1]
  auto Ds = reinterpret_cast<T(*)[BS + 1]>(smem_raw + sizeof(T) * BS * (BS + 1));
  auto Vs = reinterpret_cast<T(*)[NR]>(smem_raw + 2 * sizeof(T) * BS * (BS + 1));
  __shared__ unsigned s_I, s_known;
  const int t = threadIdx.x, r = t & (BS - 1), g = t >> 6;
  if (t == 0) {
    s_I = atomicAdd(&ctr[0], 1u);
    s_known = 0;
  }
  __syncthreads();
  const int I = (int)s_I, i0 = I * BS, i = i0 + r;
  {   // DI_I into shared memory first: the diagonal step then waits on no global load
    const T* D = DI + (size_t)I * BS * BS;
    for (int e = t; e < BS * BS; e += kThreads) Ds[e % BS][e / BS] = D[e];
  }
  const bool row_contig = (rs == 1);
  T acc[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int c = g * 4 + k;
    acc[k] = (i < n && c < nrhs) ? (T)(sc != nullptr ? sc[i] * (double)B[i + c * ldb] : (double)B[i + c * ldb])
                                 : T(0);
  }
  // prefetch of the next L block: element e = t + 256 q
  T pre[BS * BS / kThreads];
  auto fetch = [&](int J) {
#pragma unroll
    for (int q = 0; q < BS * BS / kThreads; ++q) {
      const int e = t + kThreads * q;
      const int ii = row_contig ? (e % BS) : (e / BS), jj = row_contig ? (e / BS) : (e % BS);
      pre[q] = (i0 + ii < n) ? L[(long long)(i0 + ii) * rs + (long long)(J * BS + jj) * cs] : T(0);
    }
  };
  if (I > 0) fetch(0);
  for (int J = 0; J < I; ++J) {
#pragma unroll
    for (int q = 0; q < BS * BS / kThreads; ++q) {
      const int e = t + kThreads * q;
      const int ii = row_contig ? (e % BS) : (e / BS), jj = row_contig ? (e / BS) : (e % BS);
      Ls[ii][jj] = pre[q];
    }
    if (J + 1 < I) fetch(J + 1);
    if (t == 0 && s_known < (unsigned)(J + 1)) s_known = wait_ready(&ctr[1], (unsigned)(J + 1), err, wait_limit);
    __syncthreads();
    {
      const int jj = t >> 4, c = t & 15;   // y_J into shared memory (L2 reads: written by another CTA)
      Vs[jj][c] = __ldcg(&Y[(long long)(J * BS + jj) + c * ldy]);
      const int jj2 = jj + 16;
      Vs[jj2][c] = __ldcg(&Y[(long long)(J * BS + jj2) + c * ldy]);
      Vs[jj2 + 16][c] = __ldcg(&Y[(long long)(J * BS + jj2 + 16) + c * ldy]);
      Vs[jj2 + 32][c] = __ldcg(&Y[(long long)(J * BS + jj2 + 32) + c * ldy]);
    }
    __syncthreads();
#pragma unroll 8
    for (int cc = 0; cc < BS; ++cc) {
      const T l = Ls[r][cc];
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] -= l * Vs[cc][g * 4 + k];
    }
    __syncthreads();
  }
  // y_I = DI_I acc
#pragma unroll
  for (int k = 0; k < 4; ++k) Vs[r][g * 4 + k] = acc[k];
  __syncthreads();
  T y[4] = {T(0), T(0), T(0), T(0)};
  for (int cc = 0; cc <= r; ++cc) {
    const T d = Ds[r][cc];
#pragma unroll
    for (int k = 0; k < 4; ++k) y[k] += d * Vs[cc][g * 4 + k];
  }
  if (i < n) {
#pragma unroll
    for (int k = 0; k < 4; ++k) __stcg(&Y[i + (long long)(g * 4 + k) * ldy], y[k]);
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) __stcg(&Y[i + (long long)(g * 4 + k) * ldy], T(0));
  }
  __threadfence();
  __syncthreads();
  if (t == 0) st_release(&ctr[1], (unsigned)(I + 1));
}

// Z := sc .* (L^-T Y) (type VZ, ldz), the transposed solve of trsv_fwd_kernel:
// blocks taken from the last one; block I accumulates L(J, I)^T z_J for J > I.
// ctr[1] counts finished blocks from the end.  Y and Z may alias (in place).
template <typename T, typename VZ>
__global__ void __launch_bounds__(kThreads)
    trsv_bwd_kernel(const T* __restrict__ L, long long rs, long long cs, int n, const T* __restrict__ DI,
                    const T* Y, long long ldy, const double* __restrict__ sc, VZ* Z, long long ldz, T* Zt,
                    int nrhs, unsigned* ctr, int* err, int wait_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto Ls = reinterpret_cast<T(*)[BS + 1]>(smem_raw);           // Ls[c][r] = L(J*BS + c, I*BS + r)
  auto Ds = reinterpret_cast<T(*)[BS + 1]>(smem_raw + sizeof(T) * BS * (BS + 1));   // Ds[r][c] = DI_I(c, r)
  auto Vs = reinterpret_cast<T(*)[NR]>(smem_raw + 2 * sizeof(T) * BS * (BS + 1));
  __shared__ unsigned s_I, s_known;
  const int nblk = (n + BS - 1) / BS;
  const int t = threadIdx.x, r = t & (BS - 1), g = t >> 6;
  if (t == 0) {
    s_I = atomicAdd(&ctr[0], 1u);
    s_known = 0;
  }
  __syncthreads();
  const int I = nblk - 1 - (int)s_I, i0 = I * BS, i = i0 + r;
  {
    const T* D = DI + (size_t)I * BS * BS;
    for (int e = t; e < BS * BS; e += kThreads) Ds[e / BS][e % BS] = D[e];
  }
  const bool row_contig = (rs == 1);
  T acc[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) acc[k] = (i < n) ? Y[i + (long long)(g * 4 + k) * ldy] : T(0);
  T pre[BS * BS / kThreads];
  auto fetch = [&](int J) {
#pragma unroll
    for (int q = 0; q < BS * BS / kThreads; ++q) {
      const int e = t + kThreads * q;
      const int cc = row_contig ? (e % BS) : (e / BS), rr = row_contig ? (e / BS) : (e % BS);
      pre[q] = (J * BS + cc < n) ? L[(long long)(J * BS + cc) * rs + (long long)(i0 + rr) * cs] : T(0);
    }
  };
  if (I < nblk - 1) fetch(nblk - 1);
  for (int J = nblk - 1; J > I; --J) {
#pragma unroll
    for (int q = 0; q < BS * BS / kThreads; ++q) {
      const int e = t + kThreads * q;
      const int cc = row_contig ? (e % BS) : (e / BS), rr = row_contig ? (e / BS) : (e % BS);
      Ls[cc][rr] = pre[q];
    }
    if (J - 1 > I) fetch(J - 1);
    const unsigned need = (unsigned)(nblk - J);
    if (t == 0 && s_known < need) s_known = wait_ready(&ctr[1], need, err, wait_limit);
    __syncthreads();
    {
      const int jj = t >> 4, c = t & 15;
#pragma unroll
      for (int q = 0; q < 4; ++q) Vs[jj + 16 * q][c] = __ldcg(&Zt[(long long)(J * BS + jj + 16 * q) + c * ldy]);
    }
    __syncthreads();
#pragma unroll 8
    for (int cc = 0; cc < BS; ++cc) {
      const T l = Ls[cc][r];
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] -= l * Vs[cc][g * 4 + k];
    }
    __syncthreads();
  }
  // z_I = DI_I^T acc
#pragma unroll
  for (int k = 0; k < 4; ++k) Vs[r][g * 4 + k] = acc[k];
  __syncthreads();
  T z[4] = {T(0), T(0), T(0), T(0)};
  for (int cc = r; cc < BS; ++cc) {
    const T d = Ds[r][cc];
#pragma unroll
    for (int k = 0; k < 4; ++k) z[k] += d * Vs[cc][g * 4 + k];
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int c = g * 4 + k;
    __stcg(&Zt[i + (long long)c * ldy], (i < n) ? z[k] : T(0));
    if (i < n && c < nrhs) Z[i + (long long)c * ldz] = (VZ)((sc != nullptr) ? sc[i] * (double)z[k] : (double)z[k]);
  }
  __threadfence();
  __syncthreads();
  if (t == 0) st_release(&ctr[1], (unsigned)(nblk - I));
}

// ---- preconditioner: blocked triangular solves with inverted diagonal blocks -------
// M^-1 r = S F^T F S r with F = the forward solve by L (the FP32 factor), done in
// NBT-wide block steps: y_I = inv(L_II) t_I, then t_below -= L(below, I) y_I (and
// the transposed sequence backwards).  inv(L_II) is formed once per factor, so each
// step is two GEMVs that spread over the whole GPU: no step waits on a chain of
// small blocks.  FP32 throughout (it is the preconditioner); 16 right-hand sides.
constexpr int GR = 64;            // rows (gemv_n) or output columns (gemv_t) per CTA
constexpr int GMP = GR + 4;       // shared row pitch of a 64 x 64 chunk
constexpr int GVP = NR + 4;       // shared row pitch of a vector chunk

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(tc::smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async16_(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(tc::smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
constexpr int GST = 4;                                  // cp.async stages
constexpr int GSTAGE = GR * GMP + GR * GVP;             // floats per stage
constexpr size_t kGemvSmem = sizeof(float) * (GST * GSTAGE + 4 * GR * NR);

// The 4 partial 4 x 4 blocks of every thread -> out (alpha, beta), rows/columns
// [o0, o0 + 64) of the output; with a split k range (part != null) the raw sums go to
// part[o][c] of this split instead, for gemv_reduce_kernel.
__device__ __forceinline__ void gemv_finish(float (&acc)[4][4], float* Red, int ig, int cg, int ks, int o0, int m,
                                            float alpha, float beta, const float* in, float* out, long long ldv,
                                            float* part) {
  const int t = threadIdx.x;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) Red[(ks * GR + 4 * ig + i) * NR + 4 * cg + j] = acc[i][j];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int o = t & 63, c = (t >> 6) * 4 + q, r = o0 + o;
    const float sum = ((Red[(0 * GR + o) * NR + c] + Red[(1 * GR + o) * NR + c]) +
                       (Red[(2 * GR + o) * NR + c] + Red[(3 * GR + o) * NR + c]));
    if (part != nullptr) {
      part[(long long)r * NR + c] = sum;
    } else if (r < m) {
      float v = alpha * sum;
      if (beta != 0.f) v = fmaf(beta, in[r + (long long)c * ldv], v);
      out[r + (long long)c * ldv] = v;
    }
  }
}

// out(r, c) = alpha * sum_s part[s][r][c] + beta * in(r, c), the splits in order.
__global__ void gemv_reduce_kernel(const float* __restrict__ part, int nsplit, long long mp, int m, float alpha,
                                   float beta, const float* in, float* out, long long ldv) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)m * NR) return;
  const int r = (int)(e / NR), c = (int)(e % NR);
  float sum = 0.f;
  for (int q = 0; q < nsplit; ++q) sum += part[((long long)q * mp + r) * NR + c];
  float v = alpha * sum;
  if (beta != 0.f) v = fmaf(beta, in[r + (long long)c * ldv], v);
  out[r + (long long)c * ldv] = v;
}

// 16 consecutive k of the stage: thread block (ig, cg) += A4(ig rows) x V4(cg rhs).
__device__ __forceinline__ void gemv_mac(const float* Ms, const float* Vs, int ig, int cg, int ks,
                                         float (&acc)[4][4]) {
#pragma unroll
  for (int kq = 0; kq < 16; ++kq) {
    const int k = ks * 16 + kq;
    const float4 a = *reinterpret_cast<const float4*>(&Ms[k * GMP + 4 * ig]);
    const float4 b = *reinterpret_cast<const float4*>(&Vs[k * GVP + 4 * cg]);
    const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
  }
}

// v chunk k0.. (64 x 16) -> Vs[k][c], zero past kk
__device__ __forceinline__ void gemv_issue_v(float* Vs, const float* v, long long ldv, int kk, int k0) {
  const int t = threadIdx.x;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = t + kThreads * q, k = e & 63, c = e >> 6, gk = k0 + k;
    cp_async4(&Vs[k * GVP + c], v + (gk < kk ? gk + (long long)c * ldv : 0), gk < kk ? 4 : 0);
  }
}

// out(r, c) = alpha * sum_k M(r, k) v(k, c) + beta * in(r, c), r < m, k < kk.
// M: FP32 column-major (ldm a multiple of 4, 16-byte aligned columns); v / in / out:
// FP32 column-major with leading dimension ldv (in may alias out).  CTA: 64 rows;
// M and v stream through a 4-stage cp.async ring in 64-wide k chunks (each column
// segment of 64 rows = 16 pieces of 16 bytes, stored as Ms[k][row]); thread: 4 rows
// x 4 right-hand sides over a quarter of each chunk.
__global__ void __launch_bounds__(kThreads)
    gemv_n_kernel(const float* __restrict__ M, long long ldm, int m, int kk, const float* __restrict__ v,
                  float alpha, float beta, const float* in, float* out, long long ldv, int kc, float* part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* ring = reinterpret_cast<float*>(smem_raw);
  float* Red = ring + GST * GSTAGE;
  const int t = threadIdx.x, ig = t & 15, cg = (t >> 4) & 3, ks = t >> 6;
  const int r0 = blockIdx.x * GR;
  // this CTA's k range [kb, ke): split blockIdx.y of width kc (a multiple of 64)
  const int kb = blockIdx.y * kc, ke = min(kk, kb + kc);
  const int nch = (ke - kb + GR - 1) / GR;
  auto issue = [&](int ch) {
    float* Ms = ring + (ch % GST) * GSTAGE;
    float* Vs = Ms + GR * GMP;
    const int k0 = kb + ch * GR;
#pragma unroll
    for (int q = 0; q < 4; ++q) {   // 16-byte piece f of column col: rows r0 + 4f ..
      const int e = t + kThreads * q, f = e & 15, col = e >> 4, r = r0 + 4 * f, k = k0 + col;
      const float* src = M + r + (long long)k * ldm;
      int bytes = 0;
      if (k < ke && r < m) bytes = (r + 3 < m) ? 16 : 4 * (m - r);
      cp_async16_(&Ms[col * GMP + 4 * f], bytes ? src : M, bytes);
    }
    gemv_issue_v(Vs, v, ldv, ke, k0);
  };
  float acc[4][4] = {};
  for (int ch = 0; ch < GST - 1; ++ch) {
    if (ch < nch) issue(ch);
    cp_async_commit();
  }
  for (int ch = 0; ch < nch; ++ch) {
    cp_async_wait<GST - 2>();
    __syncthreads();
    if (ch + GST - 1 < nch) issue(ch + GST - 1);
    cp_async_commit();
    const float* Ms = ring + (ch % GST) * GSTAGE;
    gemv_mac(Ms, Ms + GR * GMP, ig, cg, ks, acc);
  }
  cp_async_wait<0>();
  gemv_finish(acc, Red, ig, cg, ks, r0, m, alpha, beta, in, out, ldv,
              part ? part + (long long)blockIdx.y * gridDim.x * GR * NR : nullptr);
}

// out(j, c) = alpha * sum_k M(k, j) v(k, c) + beta * in(j, c), j < m, k < kk (the
// transposed product).  CTA: 64 output columns; the chunk is transposed on its way
// into shared memory (4-byte copies, Ms[k][col]) so that a thread reads 4 columns
// with one 16-byte load.
__global__ void __launch_bounds__(kThreads)
    gemv_t_kernel(const float* __restrict__ M, long long ldm, int m, int kk, const float* __restrict__ v,
                  float alpha, float beta, const float* in, float* out, long long ldv, int kc, float* part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* ring = reinterpret_cast<float*>(smem_raw);
  float* Red = ring + GST * GSTAGE;
  const int t = threadIdx.x, jg = t & 15, cg = (t >> 4) & 3, ks = t >> 6;
  const int j0 = blockIdx.x * GR;
  const int kb = blockIdx.y * kc, ke = min(kk, kb + kc);
  const int nch = (ke - kb + GR - 1) / GR;
  auto issue = [&](int ch) {
    float* Ms = ring + (ch % GST) * GSTAGE;
    float* Vs = Ms + GR * GMP;
    const int k0 = kb + ch * GR;
#pragma unroll
    for (int q = 0; q < 16; ++q) {   // element (k, col): consecutive threads, consecutive k
      const int e = t + kThreads * q, k = e & 63, col = e >> 6, gk = k0 + k, j = j0 + col;
      const bool ok = gk < ke && j < m;
      cp_async4(&Ms[k * GMP + col], ok ? M + gk + (long long)j * ldm : M, ok ? 4 : 0);
    }
    gemv_issue_v(Vs, v, ldv, ke, k0);
  };
  float acc[4][4] = {};
  for (int ch = 0; ch < GST - 1; ++ch) {
    if (ch < nch) issue(ch);
    cp_async_commit();
  }
  for (int ch = 0; ch < nch; ++ch) {
    cp_async_wait<GST - 2>();
    __syncthreads();
    if (ch + GST - 1 < nch) issue(ch + GST - 1);
    cp_async_commit();
    const float* Ms = ring + (ch % GST) * GSTAGE;
    gemv_mac(Ms, Ms + GR * GMP, jg, cg, ks, acc);
  }
  cp_async_wait<0>();
  gemv_finish(acc, Red, jg, cg, ks, j0, m, alpha, beta, in, out, ldv,
              part ? part + (long long)blockIdx.y * gridDim.x * GR * NR : nullptr);
}

// t = (float)(s .* r) (NR columns)
__global__ void scale_in_kernel(const double* __restrict__ r, const double* __restrict__ s, int n, long long ld,
                                float* __restrict__ out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * NR;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    out[i + c * ld] = (float)(s[i] * r[i + c * ld]);
  }
}
// z = s .* (double)y
__global__ void scale_out_kernel(const float* __restrict__ y, const double* __restrict__ s, int n, long long ld,
                                 double* __restrict__ z) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * NR;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    z[i + c * ld] = s[i] * (double)y[i + c * ld];
  }
}

// dst(i, j) = src(i, j) converted, for i >= j (lower) or all (full); others zero.
template <typename S, typename D>
__global__ void convert_kernel(const S* __restrict__ src, long long lds, D* __restrict__ dst, long long ldd, int n,
                               int lower) {
  const int i = blockIdx.x * 32 + (threadIdx.x & 31);
  for (int j = blockIdx.y * 32 + (threadIdx.x >> 5); j < min(n, blockIdx.y * 32 + 32); j += 8) {
    if (i < n) dst[i + (long long)j * ldd] = (!lower || i >= j) ? (D)src[i + (long long)j * lds] : D(0);
  }
}

// ---- symmetric product A X in FP64 ----------------------------------------------

// Tile task t <-> lower tile (I, J), J <= I, row-major: t = I (I + 1) / 2 + J.
__device__ __forceinline__ void task_tile(int t, int& I, int& J) {
  int r = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while (r > 0 && r * (r + 1) / 2 > t) --r;
  while ((r + 1) * (r + 2) / 2 <= t) ++r;
  I = r;
  J = t - r * (r + 1) / 2;
}

// Each stored element of the triangle is read once: the CTA of lower tile (I, J)
// writes the partial products U(I,J) = A_IJ X_J (rows of block I) and
// V(I,J) = A_IJ^T X_I (rows of block J; on a diagonal tile only the strictly lower
// part), each SY x NR, row-major [row][rhs].  absval: |A| instead of A.
// The CTA reads its tile in the stored orientation (always whole columns): for
// lower storage T = A(I-rows, J-cols), for upper storage T = A(J-rows, I-cols) =
// A_IJ^T, and then T X and T^T X trade places.  Columns are streamed in 16-column
// chunks through a 3-stage cp.async ring, and both products run on the FP64 tensor
// cores (mma.sync m16n8k4): warp w computes T X for rows [32w, 32w + 32) and a
// partial T^T X over the same 32 rows; the 8 partials are summed in shared memory.
// FP64 tensor-bound at 16 right-hand sides (n^2 * NR FMAs for n^2 / 2 * 8 bytes).
constexpr int kSP = SY + 4;    // S row pitch (doubles): conflict-free fragment loads
constexpr int kXP = NR + 4;    // Xi row pitch
constexpr int kCP = 16 + 4;    // Xc row pitch (Xc[c][jj])
constexpr int kStages = 3;
constexpr size_t kSymvSmemBytes =
    sizeof(double) * (kStages * 16 * kSP + kStages * NR * kCP + SY * kXP + 8 * 16 * NR);

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(tc::smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(tc::smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}

__global__ void __launch_bounds__(kThreads, 1)
    symv_tiles_kernel(const double* __restrict__ a, long long lda, int upper, int n,
                      const double* __restrict__ X, long long ldx, int nrhs, int absval, int vec16,
                      double* __restrict__ U, double* __restrict__ V) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* Sr = reinterpret_cast<double*>(smem_raw);   // stage s: Sr[s][jj * kSP + ii] = T(ii, chunk col jj)
  double* Xcr = Sr + kStages * 16 * kSP;               // stage s: Xcr[s][c * kCP + jj] = X(col block + jj, c)
  double* Xi = Xcr + kStages * NR * kCP;               // Xi[ii * kXP + c] = X(row block + ii, c)
  double* Vr = Xi + SY * kXP;                          // Vr[w][jj][c]: per-warp partial T^T X
  int I, J;
  task_tile(blockIdx.x, I, J);
  const int rb = upper ? J : I, cb = upper ? I : J;   // row / column block of T
  const int i0 = rb * SY, j0 = cb * SY, t = threadIdx.x;
  const int lane = t & 31, w = t >> 5, g = lane >> 2, tq = lane & 3;
  const bool diag = (I == J);
  for (int e = t; e < SY * NR; e += kThreads) {
    const int ii = e % SY, c = e / SY, i = i0 + ii;
    Xi[ii * kXP + c] = (i < n && c < nrhs) ? X[i + (long long)c * ldx] : 0.0;
  }
  // chunk jc -> stage st: 16 columns x 256 rows of T, and the 16 x 16 block of X
  auto issue = [&](int jc, int st) {
    double* S = Sr + st * 16 * kSP;
    const int jb0 = j0 + jc * 16;
    if (vec16) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int e = t + kThreads * q;            // 16-byte piece: column e / 128, rows 2 (e % 128) ..
        const int jj = e >> 7, ii = 2 * (e & 127), i = i0 + ii, j = jb0 + jj;
        const int bytes = (j < n && i < n) ? (i + 1 < n ? 16 : 8) : 0;
        cp_async16(S + jj * kSP + ii, a + (bytes ? (long long)i + (long long)j * lda : 0), bytes);
      }
    } else {
#pragma unroll 4
      for (int q = 0; q < 16; ++q) {
        const int e = t + kThreads * q;
        const int jj = e >> 8, ii = e & 255, i = i0 + ii, j = jb0 + jj;
        const int bytes = (j < n && i < n) ? 8 : 0;
        cp_async8(S + jj * kSP + ii, a + (bytes ? (long long)i + (long long)j * lda : 0), bytes);
      }
    }
    if (t < NR * 8) {   // X block: 16 columns c of 16 rows each, 16-byte pieces (2 rows)
      double* Xc = Xcr + st * NR * kCP;
      const int c = t >> 3, jj = 2 * (t & 7), j = jb0 + jj;
      if (((ldx & 1) == 0) && (((uintptr_t)X & 15) == 0)) {
        const int bytes = (c < nrhs && j < n) ? (j + 1 < n ? 16 : 8) : 0;
        cp_async16(Xc + c * kCP + jj, X + (bytes ? (long long)j + (long long)c * ldx : 0), bytes);
      } else {
        const int b0 = (c < nrhs && j < n) ? 8 : 0, b1 = (c < nrhs && j + 1 < n) ? 8 : 0;
        cp_async8(Xc + c * kCP + jj, X + (b0 ? (long long)j + (long long)c * ldx : 0), b0);
        cp_async8(Xc + c * kCP + jj + 1, X + (b1 ? (long long)j + 1 + (long long)c * ldx : 0), b1);
      }
    }
  };
  double u[2][2][4];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int e = 0; e < 4; ++e) u[m][q][e] = 0.0;
  double* Uo = (upper ? V : U) + (size_t)blockIdx.x * SY * NR;   // T X
  double* Vo = (upper ? U : V) + (size_t)blockIdx.x * SY * NR;   // T^T X
  const int r0 = 32 * w;   // this warp's rows of the tile
  constexpr int NCH = SY / 16;
  issue(0, 0);
  cp_async_commit();
  issue(1, 1);
  cp_async_commit();
  for (int jc = 0; jc < NCH; ++jc) {
    const int st = jc % kStages;
    cp_async_wait<kStages - 2>();   // chunk jc has landed (this thread's copies)
    __syncthreads();                // ... everyone's; and stage (jc + 2) % 3 is free
    double* S = Sr + st * 16 * kSP;
    const double* Xc = Xcr + st * NR * kCP;
    if (diag || absval) {   // keep the stored triangle only (the other one may hold anything)
      for (int e = t; e < 16 * SY; e += kThreads) {
        const int jj = e >> 8, ii = e & 255, col = jc * 16 + jj;
        double v = S[jj * kSP + ii];
        if (diag && (upper ? ii > col : ii < col)) v = 0.0;
        if (absval) v = fabs(v);
        S[jj * kSP + ii] = v;
      }
      __syncthreads();
    }
    if (jc + 2 < NCH) issue(jc + 2, (jc + 2) % kStages);
    cp_async_commit();
    // T X: 2 m16 tiles x 2 n8 tiles x 4 k4 steps
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      const double* Sk = S + (4 * ks + tq) * kSP + r0 + g;
      const double b0 = Xc[g * kCP + 4 * ks + tq], b1 = Xc[(8 + g) * kCP + 4 * ks + tq];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const double a0 = Sk[16 * m], a1 = Sk[16 * m + 8];
        cuchol::dmma::dmma_16x8x4(u[m][0], a0, a1, b0);
        cuchol::dmma::dmma_16x8x4(u[m][1], a0, a1, b1);
      }
    }
    // partial T^T X over rows r0..r0+31 (on a diagonal tile without the diagonal)
    double v[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
#pragma unroll
    for (int ks = 0; ks < 8; ++ks) {
      const int ii = r0 + 4 * ks + tq;
      double a0 = S[g * kSP + ii], a1 = S[(g + 8) * kSP + ii];
      if (diag) {
        if (ii == jc * 16 + g) a0 = 0.0;
        if (ii == jc * 16 + g + 8) a1 = 0.0;
      }
      const double b0 = Xi[ii * kXP + g], b1 = Xi[ii * kXP + 8 + g];
      cuchol::dmma::dmma_16x8x4(v[0], a0, a1, b0);
      cuchol::dmma::dmma_16x8x4(v[1], a0, a1, b1);
    }
    // C fragment: (row g, cols 2tq, 2tq+1) and (row g + 8, same cols) of each n8 tile
    double* Vw = Vr + w * 16 * NR;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      Vw[g * NR + 8 * q + 2 * tq] = v[q][0];
      Vw[g * NR + 8 * q + 2 * tq + 1] = v[q][1];
      Vw[(g + 8) * NR + 8 * q + 2 * tq] = v[q][2];
      Vw[(g + 8) * NR + 8 * q + 2 * tq + 1] = v[q][3];
    }
    __syncthreads();
    {
      double sum = 0.0;   // thread t: output (jj = t / 16, c = t % 16), warps in order
#pragma unroll
      for (int k = 0; k < 8; ++k) sum += Vr[k * 16 * NR + t];
      Vo[(jc * 16) * NR + t] = sum;
    }
  }
  cp_async_wait<0>();
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int row = r0 + 16 * m + g, col = 8 * q + 2 * tq;
      Uo[row * NR + col] = u[m][q][0];
      Uo[row * NR + col + 1] = u[m][q][1];
      Uo[(row + 8) * NR + col] = u[m][q][2];
      Uo[(row + 8) * NR + col + 1] = u[m][q][3];
    }
}

// Y_K = alpha * (sum_{J <= K} U(K,J) + sum_{I >= K} V(I,K)) + beta * B_K, summed in
// a fixed order (deterministic).  One CTA per SY-row block, thread = row.
// B may alias Y; ldy/ldb columns, only the first nrhs columns are written.
__global__ void __launch_bounds__(kThreads)
    symv_reduce_kernel(const double* __restrict__ U, const double* __restrict__ V, int n, int ntile, double alpha,
                       double beta, const double* B, long long ldb, double* Y, long long ldy, int nrhs) {
  const int K = blockIdx.x, t = threadIdx.x, i = K * SY + t;
  double sum[NR];
#pragma unroll
  for (int c = 0; c < NR; ++c) sum[c] = 0.0;
  for (int J = 0; J <= K; ++J) {
    const double* p = U + ((size_t)(K * (K + 1) / 2 + J) * SY + t) * NR;
#pragma unroll
    for (int c = 0; c < NR; ++c) sum[c] += p[c];
  }
  for (int I = K; I < ntile; ++I) {
    const double* p = V + ((size_t)(I * (I + 1) / 2 + K) * SY + t) * NR;
#pragma unroll
    for (int c = 0; c < NR; ++c) sum[c] += p[c];
  }
  if (i >= n) return;
#pragma unroll
  for (int c = 0; c < NR; ++c) {
    if (c < nrhs) {
      double y = alpha * sum[c];
      if (beta != 0.0) y += beta * B[i + (long long)c * ldb];
      Y[i + (long long)c * ldy] = y;
    }
  }
}

// ---- PCG vector kernels (n x NR, column-major, leading dimension ld) ------------------
// Deterministic reductions: each CTA writes per-RHS partials part[blockIdx.x][NR];
// the kernel that consumes them sums all partials in the same order.
constexpr int kVecBlocks = 256;

__device__ __forceinline__ void block_sum16(double (&v)[NR], double* sh /* [kThreads][NR+1] */) {
  const int t = threadIdx.x;
#pragma unroll
  for (int c = 0; c < NR; ++c) sh[t * (NR + 1) + c] = v[c];
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
#pragma unroll
      for (int c = 0; c < NR; ++c) sh[t * (NR + 1) + c] += sh[(t + s) * (NR + 1) + c];
    }
    __syncthreads();
  }
}
__device__ __forceinline__ void block_max16(double (&v)[NR], double* sh) {
  const int t = threadIdx.x;
#pragma unroll
  for (int c = 0; c < NR; ++c) sh[t * (NR + 1) + c] = v[c];
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
#pragma unroll
      for (int c = 0; c < NR; ++c) sh[t * (NR + 1) + c] = fmax(sh[t * (NR + 1) + c], sh[(t + s) * (NR + 1) + c]);
    }
    __syncthreads();
  }
}

// part[b][c] = sum over this CTA's rows of a(i, c) * b(i, c)
__global__ void __launch_bounds__(kThreads) dot_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                                       int n, long long ld, double* __restrict__ part) {
  __shared__ double sh[kThreads * (NR + 1)];
  double v[NR];
#pragma unroll
  for (int c = 0; c < NR; ++c) v[c] = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
#pragma unroll
    for (int c = 0; c < NR; ++c) v[c] = fma(a[i + c * ld], b[i + c * ld], v[c]);
  }
  block_sum16(v, sh);
  if (threadIdx.x < NR) part[blockIdx.x * NR + threadIdx.x] = sh[threadIdx.x];
}

__device__ __forceinline__ double sum_parts(const double* part, int nparts, int c) {
  double s = 0.0;
  for (int b = 0; b < nparts; ++b) s += part[b * NR + c];
  return s;
}

// alpha_c = rz_c / (p_c . q_c); x += alpha p; r -= alpha q; partial max |r|, max |x|
// into part_norm[b][0..NR) and [NR..2NR).
__global__ void __launch_bounds__(kThreads)
    update_xr_kernel(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                     const double* __restrict__ q, int n, long long ld, const double* __restrict__ part_pq,
                     const double* __restrict__ rz, double* __restrict__ part_norm) {
  __shared__ double alpha[NR];
  __shared__ double sh[kThreads * (NR + 1)];
  if (threadIdx.x < NR) {
    const int c = threadIdx.x;
    const double pq = sum_parts(part_pq, kVecBlocks, c);
    alpha[c] = (pq > 0.0 && rz[c] > 0.0) ? rz[c] / pq : 0.0;
  }
  __syncthreads();
  double rm[NR], xm[NR];
#pragma unroll
  for (int c = 0; c < NR; ++c) rm[c] = xm[c] = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
#pragma unroll
    for (int c = 0; c < NR; ++c) {
      const double xv = fma(alpha[c], p[i + c * ld], x[i + c * ld]);
      const double rv = fma(-alpha[c], q[i + c * ld], r[i + c * ld]);
      x[i + c * ld] = xv;
      r[i + c * ld] = rv;
      rm[c] = fmax(rm[c], fabs(rv));
      xm[c] = fmax(xm[c], fabs(xv));
    }
  }
  block_max16(rm, sh);
  if (threadIdx.x < NR) part_norm[blockIdx.x * 2 * NR + threadIdx.x] = sh[threadIdx.x];
  __syncthreads();
  block_max16(xm, sh);
  if (threadIdx.x < NR) part_norm[blockIdx.x * 2 * NR + NR + threadIdx.x] = sh[threadIdx.x];
}

// partial max |a(:, c)| and max |b(:, c)| (b may be null)
__global__ void __launch_bounds__(kThreads) norms_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                                         int n, long long ld, double* __restrict__ part_norm) {
  __shared__ double sh[kThreads * (NR + 1)];
  double am[NR], bm[NR];
#pragma unroll
  for (int c = 0; c < NR; ++c) am[c] = bm[c] = 0.0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
#pragma unroll
    for (int c = 0; c < NR; ++c) {
      am[c] = fmax(am[c], fabs(a[i + c * ld]));
      if (b != nullptr) bm[c] = fmax(bm[c], fabs(b[i + c * ld]));
    }
  }
  block_max16(am, sh);
  if (threadIdx.x < NR) part_norm[blockIdx.x * 2 * NR + threadIdx.x] = sh[threadIdx.x];
  __syncthreads();
  block_max16(bm, sh);
  if (threadIdx.x < NR) part_norm[blockIdx.x * 2 * NR + NR + threadIdx.x] = sh[threadIdx.x];
}

// out[0..2NR) = max over the partials (one CTA)
__global__ void norms_final_kernel(const double* __restrict__ part_norm, int nparts, double* __restrict__ out) {
  const int c = threadIdx.x;
  if (c >= 2 * NR) return;
  double m = 0.0;
  for (int b = 0; b < nparts; ++b) m = fmax(m, part_norm[b * 2 * NR + c]);
  out[c] = m;
}

// rz_new = sum of part_rz; beta = rz_new / rz_old (0 when restart or rz_old == 0);
// p = z + beta p.  Block 0 stores rz_new.
__global__ void __launch_bounds__(kThreads)
    update_p_kernel(double* __restrict__ p, const double* __restrict__ z, int n, long long ld,
                    const double* __restrict__ part_rz, const double* __restrict__ rz_old,
                    double* __restrict__ rz_new, int restart) {
  __shared__ double beta[NR];
  if (threadIdx.x < NR) {
    const int c = threadIdx.x;
    const double rn = sum_parts(part_rz, kVecBlocks, c);
    beta[c] = (!restart && rz_old[c] > 0.0) ? rn / rz_old[c] : 0.0;
    if (blockIdx.x == 0) rz_new[c] = rn;
  }
  __syncthreads();
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
#pragma unroll
    for (int c = 0; c < NR; ++c) p[i + c * ld] = fma(beta[c], p[i + c * ld], z[i + c * ld]);
  }
}

// dst (ld) = src (lds) for columns < ncols, zero for the rest of the NR columns
__global__ void load_cols_kernel(const double* __restrict__ src, long long lds, int ncols, int n,
                                 double* __restrict__ dst, long long ld) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * NR;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    dst[i + c * ld] = (c < ncols) ? src[i + c * lds] : 0.0;
  }
}
__global__ void store_cols_kernel(const double* __restrict__ src, long long ld, int ncols, int n,
                                  double* __restrict__ dst, long long ldd) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)n * ncols;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    dst[i + c * ldd] = src[i + c * ld];
  }
}

}  // namespace mx
}  // namespace

// ---- host side ------------------------------------------------------------------

struct __cucholmixed_st {
  CULAPACKhandle h;
  int precision;              // CUCHOL_MIXED_BF16 or CUCHOL_MIXED_TF32
  int n;
  const double* A;            // the caller's matrix (read by every residual)
  long long rs, cs;           // its logical lower view
  float* W;                   // FP32 factor of S A S + shift I (lower, ldw)
  long long ldw;
  double* s;                  // the scaling S
  float* Dinv;                // inverses of W's NBT x NBT diagonal blocks (ld NBT)
  float* dtmp;                // doubling scratch (n * NBT / 4)
  float* gpart;               // split-k partial sums of the preconditioner GEMVs
  double anorm;               // |A|_inf
  double shift;               // shift of the factor that succeeded
  double shift_request;       // caller's shift (< 0: automatic)
  long long ld;               // rows of the work vectors
  double *x, *r, *z, *p, *q, *b;
  float *t, *y, *zf;          // preconditioner vectors (FP32)
  double *U, *V;              // symmetric-product partials
  double *part, *part_norm, *rz, *norms;
  double* h_norms;            // pinned mirror of norms
  unsigned* ctr;              // triangular-solve counters
  int* err;                   // a bounded wait gave up
};

namespace {
namespace mx {

inline int ntile_of(int n) { return (n + SY - 1) / SY; }
constexpr size_t kSymvSmem = kSymvSmemBytes;

template <typename T>
CUresult block_inverse(const T* L, long long rs, long long cs, int n, T* DI, cudaStream_t s) {
  const size_t smem = 2 * sizeof(T) * BS * (BS + 1);
  static bool attr = false;
  if (!attr) {
    CUCHOL_CHECK(cudaFuncSetAttribute(block_inverse_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    attr = true;
  }
  block_inverse_kernel<T><<<(n + BS - 1) / BS, BS, smem, s>>>(L, rs, cs, n, DI);
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

// Y = alpha A X + beta B for the symmetric A (one triangle, lower view rs, cs).
CUresult symv(const double* A, long long rs, long long cs, int n, const double* X, long long ldx, int nrhs,
              int absval, double alpha, double beta, const double* B, long long ldb, double* Y, long long ldy,
              double* U, double* V, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    CUCHOL_CHECK(cudaFuncSetAttribute(symv_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kSymvSmem));
    attr = true;
  }
  const int T = ntile_of(n);
  const int upper = (rs != 1);
  const long long lda = upper ? rs : cs;
  const int vec16 = ((lda & 1) == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0);
  symv_tiles_kernel<<<T * (T + 1) / 2, kThreads, kSymvSmem, s>>>(A, lda, upper, n, X, ldx, nrhs, absval, vec16, U,
                                                                  V);
  CUCHOL_CHECK(cudaGetLastError());
  symv_reduce_kernel<<<T, kThreads, 0, s>>>(U, V, n, T, alpha, beta, B, ldb, Y, ldy, nrhs);
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

template <typename T>
constexpr size_t trsv_smem() { return sizeof(T) * (2 * BS * (BS + 1) + BS * NR); }

// Opt in to the triangular solves' shared memory (above 48 KB for FP64).
template <typename T, typename V>
CUresult trsv_attr() {
  static bool done = false;
  if (!done) {
    CUCHOL_CHECK(cudaFuncSetAttribute(trsv_fwd_kernel<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)trsv_smem<T>()));
    CUCHOL_CHECK(cudaFuncSetAttribute(trsv_bwd_kernel<T, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)trsv_smem<T>()));
    done = true;
  }
  return CUDA_SUCCESS;
}

// Z = S F^T F S R (the preconditioner; F = forward solve by the FP32 factor in
// NBT-wide steps with the inverted diagonal blocks), 16 columns.
CUresult precond(CUcholMixed p, const double* R, double* Z, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    CUCHOL_CHECK(cudaFuncSetAttribute(gemv_n_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemvSmem));
    CUCHOL_CHECK(cudaFuncSetAttribute(gemv_t_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemvSmem));
    attr = true;
  }
  const int n = p->n;
  const long long ld = p->ld, ldw = p->ldw;
  const int nT = (n + NBT - 1) / NBT, vb = 4 * p->h->num_sms;
  // one GEMV; with fewer than two CTAs per SM the k range is split (chunks of 256 or
  // more) and the partial sums reduced in order by a second launch
  auto gemv = [&](bool trans, const float* M, long long ldm, int m, int kk, const float* v, float alpha,
                  float beta, const float* in, float* out) -> CUresult {
    const int blocks = (m + GR - 1) / GR, want = 2 * p->h->num_sms;
    int split = 1;
    if (blocks < want) split = std::max(1, std::min((want + blocks - 1) / blocks, kk / 256));
    const int kc = (int)round_up((size_t)((kk + split - 1) / split), GR);
    split = (kk + kc - 1) / kc;
    float* part = split > 1 ? p->gpart : nullptr;
    const dim3 grid(blocks, split);
    if (trans)
      gemv_t_kernel<<<grid, kThreads, kGemvSmem, s>>>(M, ldm, m, kk, v, alpha, beta, in, out, ld, kc, part);
    else
      gemv_n_kernel<<<grid, kThreads, kGemvSmem, s>>>(M, ldm, m, kk, v, alpha, beta, in, out, ld, kc, part);
    CUCHOL_CHECK(cudaGetLastError());
    ++p->h->launches;
    if (split > 1) {
      gemv_reduce_kernel<<<(m * NR + 255) / 256, 256, 0, s>>>(part, split, (long long)blocks * GR, m, alpha, beta,
                                                              in, out, ld);
      CUCHOL_CHECK(cudaGetLastError());
      ++p->h->launches;
    }
    return CUDA_SUCCESS;
  };
  scale_in_kernel<<<vb, 256, 0, s>>>(R, p->s, n, ld, p->t);
  CUCHOL_CHECK(cudaGetLastError());
  for (int I = 0; I < nT; ++I) {
    const int b0 = I * NBT, bI = std::min(NBT, n - b0), rest = n - b0 - bI;
    const float* D = p->Dinv + (size_t)I * NBT * NBT;
    CUCHOL_CHECK_CU(gemv(false, D, NBT, bI, bI, p->t + b0, 1.f, 0.f, nullptr, p->y + b0));
    if (rest > 0)
      CUCHOL_CHECK_CU(gemv(false, p->W + (b0 + bI) + (long long)b0 * ldw, ldw, rest, bI, p->y + b0, -1.f, 1.f,
                           p->t + b0 + bI, p->t + b0 + bI));
  }
  for (int I = nT - 1; I >= 0; --I) {
    const int b0 = I * NBT, bI = std::min(NBT, n - b0);
    const float* D = p->Dinv + (size_t)I * NBT * NBT;
    CUCHOL_CHECK_CU(gemv(true, D, NBT, bI, bI, p->y + b0, 1.f, 0.f, nullptr, p->zf + b0));
    if (b0 > 0) CUCHOL_CHECK_CU(gemv(true, p->W + b0, ldw, b0, bI, p->zf + b0, -1.f, 1.f, p->y, p->y));
  }
  scale_out_kernel<<<vb, 256, 0, s>>>(p->zf, p->s, n, ld, Z);
  CUCHOL_CHECK(cudaGetLastError());
  p->h->launches += 2;
  return CUDA_SUCCESS;
}

// C := C + alpha Q(a0 + i) Q(b0 + j)^T (alpha = -1 in the factor) on the lower tiles of an
// m x ncols FP32 region whose
// top-left element is on the diagonal; Q k-major (q_rows x k used, row pitch ldq).
template <typename Op>
CUresult tc_update(CULAPACKhandle h, const Op* q, long long ldq, int q_rows, int k, int a0, int b0, float* c,
                   long long ldc, int m, int ncols, cudaStream_t s, const int* stop, float alpha = -1.f) {
  if (m <= 0 || ncols <= 0 || k <= 0) return CUDA_SUCCESS;
  EncodeTiledFn fn = encode_tiled();
  if (fn == nullptr) return CUDA_ERROR_NOT_SUPPORTED;
  CUtensorMap mq, mc;
  const cuuint32_t es[2] = {1, 1};
  {
    const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)q_rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ldq * sizeof(Op)};
    const cuuint32_t box[2] = {(cuuint32_t)tc::OpKind<Op>::BK, (cuuint32_t)tc::BM};
    const CUtensorMapDataType dt = sizeof(Op) == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    if (fn(&mq, dt, 2, const_cast<Op*>(q), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS)
      return CUDA_ERROR_INVALID_VALUE;
  }
  {
    const cuuint64_t dims[2] = {(cuuint64_t)m, (cuuint64_t)ncols};
    const cuuint64_t strides[1] = {(cuuint64_t)ldc * sizeof(float)};
    const cuuint32_t box[2] = {32, 32};
    if (fn(&mc, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, c, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
        CUDA_SUCCESS)
      return CUDA_ERROR_INVALID_VALUE;
  }
  tc::Params prm{};
  prm.m = m;
  prm.n = ncols;
  prm.k = k;
  prm.a_row0 = a0;
  prm.b_row0 = b0;
  prm.alpha = alpha;
  prm.lower_only = 1;
  prm.tiles_m = (m + tc::BM - 1) / tc::BM;
  prm.tiles_n = (ncols + tc::BN - 1) / tc::BN;
  prm.err = h->d_words + 3;
  const int tiles = prm.tiles_n * (prm.tiles_n + 1) / 2 + (prm.tiles_m - prm.tiles_n) * prm.tiles_n;
  static bool attr = false;
  if (!attr) {
    CUCHOL_CHECK(cudaFuncSetAttribute(tc::update_kernel<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      tc::SMEM_BYTES));
    attr = true;
  }
  tc::update_kernel<Op><<<tiles, tc::THREADS, tc::SMEM_BYTES, s>>>(mq, mq, mc, prm, stop);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

// Blocked Cholesky of the FP32 matrix W (lower, ldw) with FP64 diagonal blocks, FP32
// panel solves and tensor-core trailing updates in Op; schedule as ?potrf.
// *info = first failing column (1-based) or 0.
// The FP32 inverse of every 128-wide diagonal block is left in dinv (the NBT-block
// store of the plan, ld NBT) at its place in its NBT-wide block.
template <typename Op>
CUresult mixed_factor(CULAPACKhandle h, int n, float* W, long long ldw, long* info) {
  using Smem = DiagSmem<double, SB>;
  cudaStream_t sp = h->s_panel, su = h->s_update;
  int* d_info = h->d_words;
  const long long ldq = OB;
  const size_t rows = round_up((size_t)n, 128) + 128;
  const size_t small = round_up(sizeof(double) * SB * SB, 256);
  const size_t qbytes = round_up(sizeof(Op) * rows * ldq, 256);
  CUCHOL_CHECK_CU(ensure_workspace(h, small + 2 * qbytes));
  char* ws = static_cast<char*>(h->ws);
  double* D = reinterpret_cast<double*>(ws);
  Op* Q[2] = {reinterpret_cast<Op*>(ws + small), reinterpret_cast<Op*>(ws + small + qbytes)};
  static bool attr = false;
  if (!attr) {
    CUCHOL_CHECK(cudaFuncSetAttribute(trsm_rows_kernel<float, float, double, Op, OUT_ROUND>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_rows_smem<float>()));
    attr = true;
  }

  CUCHOL_CHECK_CU(set_smem<double>((const void*)diag_factor_kernel<double, SB, kDiagThreads2>, Smem::bytes));
  CUCHOL_CHECK(cudaMemsetAsync(d_info, 0, sizeof(int), sp));
  CUCHOL_CHECK(cudaMemsetAsync(h->d_logdet, 0, sizeof(double), sp));
  CUCHOL_CHECK(cudaEventRecord(h->ev_panel, sp));
  CUCHOL_CHECK(cudaStreamWaitEvent(su, h->ev_panel, 0));
  CUCHOL_CHECK(cudaEventRecord(h->ev_update, su));
  auto at = [&](long long i, long long j) { return W + i + j * ldw; };

  for (int j = 0, step = 0; j < n; j += OB, ++step) {
    const int jB = std::min(OB, n - j);
    const int m = n - j - jB;
    Op* Qj = Q[step & 1];
    const int q_rows = n - j - SB;   // P / Q row r = global row j + SB + r
    for (int s0 = 0; s0 < jB; s0 += SB) {
      const int c = j + s0, jb = std::min(SB, j + jB - c), mr = n - c - jb;
      diag_in_kernel<<<jb, SB, 0, sp>>>(at(c, c), ldw, jb, D, d_info);
      diag_factor_kernel<double, SB, kDiagThreads2><<<1, kDiagThreads2, Smem::bytes, sp>>>(
          D, 1, SB, jb, nullptr, SB, c, d_info, h->d_logdet);
      diag_out_kernel<<<jb, SB, 0, sp>>>(D, jb, at(c, c), ldw, d_info);
      h->launches += 3;
      CUCHOL_CHECK(cudaGetLastError());
      if (mr == 0) break;
      // panel rows c + jb .. n-1 solved in place; they are Q rows s0 .., columns s0 ..
      Op* Qs = Qj + (long long)s0 * ldq + s0;
      trsm_rows_kernel<float, float, double, Op, OUT_ROUND><<<(mr + 63) / 64, kThreads, trsm_rows_smem<float>(), sp>>>(
          at(c + jb, c), 1, ldw, mr, jb, D, 1, SB, Qs, ldq, 1, d_info, nullptr);
      ++h->launches;
      CUCHOL_CHECK(cudaGetLastError());
      if (s0 + SB < jB)   // the outer block's remaining columns by this sub-panel
        CUCHOL_CHECK_CU(tc_update<Op>(h, Qs, ldq, q_rows - s0, jb, 0, 0, at(c + jb, c + jb), ldw, mr,
                                      jB - s0 - SB, sp, d_info));
    }
    CUCHOL_CHECK(cudaEventRecord(h->ev_panel, sp));
    if (m == 0) break;
    // P / Q rows from global row j + OB: all sub-panels' columns (k = jB)
    const int jB2 = std::min(OB, m);
    const Op* Qt = Qj + (long long)(OB - SB) * ldq;
    const int t_rows = q_rows - (OB - SB);
    CUCHOL_CHECK(cudaStreamWaitEvent(sp, h->ev_update, 0));
    CUCHOL_CHECK_CU(tc_update<Op>(h, Qt, ldq, t_rows, jB, 0, 0, at(j + OB, j + OB), ldw, m, jB2, sp, d_info));
    CUCHOL_CHECK(cudaStreamWaitEvent(su, h->ev_panel, 0));
    if (m > jB2)
      CUCHOL_CHECK_CU(tc_update<Op>(h, Qt, ldq, t_rows, jB, jB2, jB2, at(j + OB + jB2, j + OB + jB2), ldw, m - jB2,
                                    m - jB2, su, d_info));
    CUCHOL_CHECK(cudaEventRecord(h->ev_update, su));
  }
  CUCHOL_CHECK(cudaEventRecord(h->ev_update, su));
  CUCHOL_CHECK(cudaStreamWaitEvent(sp, h->ev_update, 0));
  CUCHOL_CHECK(cudaMemcpyAsync(h->h_words, d_info, 4 * sizeof(int), cudaMemcpyDeviceToHost, sp));
  CUCHOL_CHECK(cudaStreamSynchronize(sp));
  CUCHOL_CHECK_CU(check_engine(h));
  *info = h->h_words[0];
  return CUDA_SUCCESS;
}

void free_mixed(CUcholMixed p) {
  if (p == nullptr) return;
  cudaFree(p->W);
  cudaFree(p->s);
  cudaFree(p->Dinv);
  cudaFree(p->dtmp);
  cudaFree(p->gpart);
  cudaFree(p->x);
  cudaFree(p->t);
  cudaFree(p->U);
  cudaFree(p->V);
  cudaFree(p->part);
  cudaFree(p->ctr);
  cudaFreeHost(p->h_norms);
  delete p;
}

// Largest column max |v(:, c)| for c < 2 NR of the partials -> host (synchronises s).
CUresult fetch_norms(CUcholMixed p, cudaStream_t s) {
  norms_final_kernel<<<1, 2 * NR, 0, s>>>(p->part_norm, kVecBlocks, p->norms);
  CUCHOL_CHECK(cudaGetLastError());
  CUCHOL_CHECK(cudaMemcpyAsync(p->h_norms, p->norms, 2 * NR * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUCHOL_CHECK(cudaStreamSynchronize(s));
  return CUDA_SUCCESS;
}

// The doubling levels of the NBT-block inverses (see mixed_refactor); the products
// B inv(A) of one level (at most n * NBT / 4 elements) go to the plan's scratch.
CUresult dinv_doubling(CUcholMixed p, cudaStream_t s) {
  const int n = p->n, nT = (n + NBT - 1) / NBT;
  const long long ldw = p->ldw;
  for (int sz = SB; sz < NBT; sz *= 2) {
    std::vector<GemmProblem<float>> first, second;
    float* tmp = p->dtmp;
    for (int I = 0; I < nT; ++I) {
      const int b0 = I * NBT, bI = std::min(NBT, n - b0);
      float* D = p->Dinv + (size_t)I * NBT * NBT;
      for (int o = 0; o + sz < bI; o += 2 * sz) {
        const int cs = std::min(sz, bI - o - sz);
        GemmProblem<float> t1 = problem<float>();   // T = B inv(A), cs x sz
        t1.a = p->W + (b0 + o + sz) + (long long)(b0 + o) * ldw; t1.a_rs = 1; t1.a_ks = ldw;
        t1.b = D + o + (long long)o * NBT; t1.b_rs = NBT; t1.b_ks = 1;
        t1.c = tmp; t1.c_rs = 1; t1.c_cs = cs;
        t1.m = cs; t1.n = sz; t1.k = sz;
        GemmProblem<float> t2 = problem<float>();   // X = -inv(C) T
        t2.a = D + (o + sz) + (long long)(o + sz) * NBT; t2.a_rs = 1; t2.a_ks = NBT;
        t2.b = tmp; t2.b_rs = cs; t2.b_ks = 1;
        t2.c = D + (o + sz) + (long long)o * NBT; t2.c_rs = 1; t2.c_cs = NBT;
        t2.m = cs; t2.n = sz; t2.k = cs;
        t2.alpha = -1.f;
        first.push_back(t1);
        second.push_back(t2);
        tmp += (size_t)cs * sz;
      }
    }
    CUCHOL_CHECK_CU(gemm_group<float>(p->h, first, s, nullptr));
    CUCHOL_CHECK_CU(gemm_group<float>(p->h, second, s, nullptr));
  }
  return CUDA_SUCCESS;
}

// Scale, |A|_inf and the low-precision factor of the plan's A (its current values).
template <typename Op>
CUresult mixed_refactor(CUcholMixed p, long* info) {
  CULAPACKhandle h = p->h;
  const int n = p->n;
  cudaStream_t sp = h->s_panel;
  // scaling; a non-positive diagonal entry ends the attempt (info = its row)
  int* bad = h->d_words + 4;
  CUCHOL_CHECK(cudaMemsetAsync(bad, 0, sizeof(int), sp));
  scale_kernel<<<(n + 255) / 256, 256, 0, sp>>>(p->A, p->rs + p->cs, n, p->s, bad);
  CUCHOL_CHECK(cudaGetLastError());
  CUCHOL_CHECK(cudaMemcpyAsync(h->h_words + 4, bad, sizeof(int), cudaMemcpyDeviceToHost, sp));
  CUCHOL_CHECK(cudaStreamSynchronize(sp));
  if (h->h_words[4] != 0) {
    std::vector<double> d(n);
    CUCHOL_CHECK(cudaMemcpy2D(d.data(), sizeof(double), p->A, (p->rs + p->cs) * sizeof(double), sizeof(double), n,
                              cudaMemcpyDeviceToHost));
    long k = 0;
    while (k < n && d[k] > 0.0) ++k;
    *info = k + 1;
    return CUDA_SUCCESS;
  }
  // |A|_inf = max row sum of |A| (x is zero: column 0 set to ones)
  CUCHOL_CHECK(cudaMemsetAsync(p->x, 0, sizeof(double) * p->ld * NR, sp));
  {
    std::vector<double> ones(n, 1.0);
    CUCHOL_CHECK(cudaMemcpyAsync(p->x, ones.data(), sizeof(double) * n, cudaMemcpyHostToDevice, sp));
    CUCHOL_CHECK_CU(symv(p->A, p->rs, p->cs, n, p->x, p->ld, 1, 1, 1.0, 0.0, nullptr, 0, p->r, p->ld, p->U, p->V,
                         sp));
    CUCHOL_CHECK(cudaMemsetAsync(p->r + p->ld, 0, sizeof(double) * p->ld * (NR - 1), sp));
    norms_kernel<<<kVecBlocks, kThreads, 0, sp>>>(p->r, nullptr, n, p->ld, p->part_norm);
    CUCHOL_CHECK(cudaGetLastError());
    CUCHOL_CHECK_CU(fetch_norms(p, sp));
    p->anorm = p->h_norms[0];
  }
  // factor S A S + shift I; on a breakdown retry with 8x the shift (automatic mode)
  const double u = (sizeof(Op) == 2) ? 0x1p-8 : 0x1p-11;
  const double shift_in = p->shift_request;
  double shift = shift_in >= 0.0 ? shift_in : u / 16;
  long finfo = 0;
  const int nT = (n + NBT - 1) / NBT;
  for (int attempt = 0; attempt < (shift_in >= 0.0 ? 1 : 4); ++attempt, shift *= 8.0) {
    dim3 g((n + 31) / 32, (n + 31) / 32);
    build_kernel<<<g, 256, 0, sp>>>(p->A, p->rs, p->cs, n, p->s, (float)shift, p->W, p->ldw);
    CUCHOL_CHECK(cudaGetLastError());
    CUCHOL_CHECK_CU(mixed_factor<Op>(h, n, p->W, p->ldw, &finfo));
    p->shift = shift;
    if (finfo == 0) break;
  }
  if (finfo != 0) {
    *info = finfo;
    return CUDA_SUCCESS;
  }
  // inverses of the NBT-wide diagonal blocks of the factor: the 128-wide diagonal
  // blocks inverted in place (one CTA each), then recursive doubling
  //   inv([A 0; B C]) = [inv(A) 0; -inv(C) B inv(A), inv(C)]
  // with one grouped launch per level and product, all NBT-blocks together (FP32).
  CUCHOL_CHECK(cudaMemsetAsync(p->Dinv, 0, sizeof(float) * (size_t)nT * NBT * NBT, sp));
  CUCHOL_CHECK_CU(set_smem<float>((const void*)diag_invert_kernel<float, SB, kDiagThreads2>,
                                  DiagSmem<float, SB>::bytes));
  for (int I = 0; I < nT; ++I) {
    const int b0 = I * NBT, bI = std::min(NBT, n - b0);
    float* Dn = p->Dinv + (size_t)I * NBT * NBT;
    CUCHOL_CHECK_CU(copy_view<float>(h, p->W + b0 + (long long)b0 * p->ldw, 1, p->ldw, Dn, 1, NBT, bI, bI, true, sp,
                                     nullptr));
    diag_invert_kernel<float, SB, kDiagThreads2><<<(bI + SB - 1) / SB, kDiagThreads2, DiagSmem<float, SB>::bytes,
                                                   sp>>>(Dn, 1, NBT, bI, SB, 0);
    ++h->launches;
    CUCHOL_CHECK(cudaGetLastError());
  }
  CUCHOL_CHECK_CU(dinv_doubling(p, sp));
  CUCHOL_CHECK(cudaStreamSynchronize(sp));
  *info = 0;
  return CUDA_SUCCESS;
}

template <typename Op>
CUresult mixed_create(CUcholMixed* out, CULAPACKhandle h, CBlasUplo uplo, size_t n_, CUdeviceptr A, size_t lda,
                      double shift_in, long* info) {
  const int n = (int)n_;
  auto* p = new (std::nothrow) __cucholmixed_st;
  if (p == nullptr) return CUDA_ERROR_OUT_OF_MEMORY;
  memset(p, 0, sizeof(*p));
  p->h = h;
  p->precision = (sizeof(Op) == 2) ? CUCHOL_MIXED_BF16 : CUCHOL_MIXED_TF32;
  p->n = n;
  p->A = reinterpret_cast<const double*>(A);
  const bool upper = (uplo == CBlasUpper);
  p->rs = upper ? (long long)lda : 1;
  p->cs = upper ? 1 : (long long)lda;
  p->ldw = (long long)round_up((size_t)n, 32);
  p->ld = (long long)round_up((size_t)n, SY);
  const int T = ntile_of(n);
  auto fail = [&](cudaError_t e) {
    free_mixed(p);
    return ::cuchol::report(e, "cudaMalloc", __func__, __FILE__, __LINE__);
  };
  cudaError_t e;
  if ((e = dev_malloc(&p->W, sizeof(float) * p->ldw * n)) != cudaSuccess) return fail(e);
  if ((e = dev_malloc(&p->s, sizeof(double) * n)) != cudaSuccess) return fail(e);
  const int nT = (n + NBT - 1) / NBT;
  if ((e = dev_malloc(&p->Dinv, sizeof(float) * (size_t)nT * NBT * NBT)) != cudaSuccess) return fail(e);
  if ((e = dev_malloc(&p->dtmp, sizeof(float) * (size_t)n * NBT / 4 + 256)) != cudaSuccess) return fail(e);
  // split k only when a GEMV has fewer than 2 * SMs row blocks: at most NBT / 256 splits
  const size_t gpart = (size_t)(NBT / 256) * (2 * h->num_sms + 1) * GR * NR;
  if ((e = dev_malloc(&p->gpart, sizeof(float) * gpart)) != cudaSuccess) return fail(e);
  // x r z p q b in one block, then the reduction scratch
  if ((e = dev_malloc(&p->x, sizeof(double) * 6 * p->ld * NR)) != cudaSuccess) return fail(e);
  p->r = p->x + p->ld * NR;
  p->z = p->r + p->ld * NR;
  p->p = p->z + p->ld * NR;
  p->q = p->p + p->ld * NR;
  p->b = p->q + p->ld * NR;
  if ((e = dev_malloc(&p->t, sizeof(float) * 3 * p->ld * NR)) != cudaSuccess) return fail(e);
  p->y = p->t + p->ld * NR;
  p->zf = p->y + p->ld * NR;
  const size_t ptile = (size_t)T * (T + 1) / 2 * SY * NR;
  if ((e = dev_malloc(&p->U, sizeof(double) * ptile)) != cudaSuccess) return fail(e);
  if ((e = dev_malloc(&p->V, sizeof(double) * ptile)) != cudaSuccess) return fail(e);
  if ((e = dev_malloc(&p->part, sizeof(double) * (kVecBlocks * NR + kVecBlocks * 2 * NR + 2 * NR + 2 * NR))) !=
      cudaSuccess)
    return fail(e);
  p->part_norm = p->part + kVecBlocks * NR;
  p->rz = p->part_norm + kVecBlocks * 2 * NR;
  p->norms = p->rz + 2 * NR;
  if ((e = dev_malloc(&p->ctr, 16 * sizeof(unsigned))) != cudaSuccess) return fail(e);
  p->err = reinterpret_cast<int*>(p->ctr + 8);
  if ((e = cudaMemset(p->ctr, 0, 16 * sizeof(unsigned))) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&p->h_norms, 2 * NR * sizeof(double))) != cudaSuccess) return fail(e);

  p->shift_request = shift_in;
  *out = p;
  return mixed_refactor<Op>(p, info);
}

// Preconditioned CG in FP64 on A x = b for the columns of B, 16 at a time.
CUresult mixed_solve(CUcholMixed p, int nrhs, const double* B, long long ldb, double* X, long long ldx, double tol,
                     int maxit, int* iter, double* berr) {
  cudaStream_t s = p->h->s_panel;
  const int n = p->n;
  const long long ld = p->ld;
  if (tol <= 0.0) tol = sqrt((double)n) * 0x1p-53;
  if (maxit <= 0) maxit = 100;
  int worst_it = 0;
  bool all_ok = true;
  double worst_berr = 0.0;
  CUCHOL_CHECK(cudaMemsetAsync(p->err, 0, sizeof(int), s));
  for (int g0 = 0; g0 < nrhs; g0 += NR) {
    const int nc = std::min(NR, nrhs - g0);
    load_cols_kernel<<<4 * p->h->num_sms, 256, 0, s>>>(B + (long long)g0 * ldb, ldb, nc, n, p->b, ld);
    CUCHOL_CHECK(cudaGetLastError());
    CUCHOL_CHECK(cudaMemcpyAsync(p->r, p->b, sizeof(double) * ld * NR, cudaMemcpyDeviceToDevice, s));
    CUCHOL_CHECK(cudaMemsetAsync(p->x, 0, sizeof(double) * ld * NR, s));
    norms_kernel<<<kVecBlocks, kThreads, 0, s>>>(p->b, nullptr, n, ld, p->part_norm);
    CUCHOL_CHECK(cudaGetLastError());
    CUCHOL_CHECK_CU(fetch_norms(p, s));
    double bn[NR];
    for (int c = 0; c < NR; ++c) bn[c] = p->h_norms[c];
    auto backward = [&](const double* rx, double* eta) {   // rx: [0,NR) |r|, [NR,2NR) |x|
      bool ok = true;
      for (int c = 0; c < nc; ++c) {
        const double den = p->anorm * rx[NR + c] + bn[c];
        eta[c] = den > 0.0 ? rx[c] / den : 0.0;
        if (!(eta[c] <= tol)) ok = false;
      }
      return ok;
    };
    double eta[NR] = {0};
    int it = 0, slot = 0;
    bool done = false;
    while (!done && it < maxit) {
      // (re)start from the current residual: p = z = M^-1 r
      CUCHOL_CHECK_CU(precond(p, p->r, p->z, s));
      dot_kernel<<<kVecBlocks, kThreads, 0, s>>>(p->r, p->z, n, ld, p->part);
      update_p_kernel<<<kVecBlocks, kThreads, 0, s>>>(p->p, p->z, n, ld, p->part, p->rz + slot * NR,
                                                      p->rz + (slot ^ 1) * NR, 1);
      CUCHOL_CHECK(cudaGetLastError());
      slot ^= 1;
      while (it < maxit) {
        CUCHOL_CHECK_CU(symv(p->A, p->rs, p->cs, n, p->p, ld, NR, 0, 1.0, 0.0, nullptr, 0, p->q, ld, p->U, p->V, s));
        dot_kernel<<<kVecBlocks, kThreads, 0, s>>>(p->p, p->q, n, ld, p->part);
        update_xr_kernel<<<kVecBlocks, kThreads, 0, s>>>(p->x, p->r, p->p, p->q, n, ld, p->part, p->rz + slot * NR,
                                                         p->part_norm);
        CUCHOL_CHECK(cudaGetLastError());
        CUCHOL_CHECK_CU(fetch_norms(p, s));
        ++it;
        if (backward(p->h_norms, eta)) break;
        CUCHOL_CHECK_CU(precond(p, p->r, p->z, s));
        dot_kernel<<<kVecBlocks, kThreads, 0, s>>>(p->r, p->z, n, ld, p->part);
        update_p_kernel<<<kVecBlocks, kThreads, 0, s>>>(p->p, p->z, n, ld, p->part, p->rz + slot * NR,
                                                        p->rz + (slot ^ 1) * NR, 0);
        CUCHOL_CHECK(cudaGetLastError());
        slot ^= 1;
      }
      // FP64 residual from scratch: r = b - A x
      CUCHOL_CHECK_CU(symv(p->A, p->rs, p->cs, n, p->x, ld, NR, 0, -1.0, 1.0, p->b, ld, p->r, ld, p->U, p->V, s));
      norms_kernel<<<kVecBlocks, kThreads, 0, s>>>(p->r, p->x, n, ld, p->part_norm);
      CUCHOL_CHECK(cudaGetLastError());
      CUCHOL_CHECK_CU(fetch_norms(p, s));
      done = backward(p->h_norms, eta);
    }
    store_cols_kernel<<<4 * p->h->num_sms, 256, 0, s>>>(p->x, ld, nc, n, X + (long long)g0 * ldx, ldx);
    CUCHOL_CHECK(cudaGetLastError());
    for (int c = 0; c < nc; ++c) worst_berr = std::max(worst_berr, eta[c]);
    worst_it = std::max(worst_it, it);
    if (!done) all_ok = false;
  }
  int err = 0;
  CUCHOL_CHECK(cudaMemcpyAsync(&err, p->err, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUCHOL_CHECK(cudaStreamSynchronize(s));
  if (err != 0) {
    if (errorHandler != nullptr)
      errorHandler("triangular solve wait", __func__, __FILE__, __LINE__, (int)CUDA_ERROR_LAUNCH_TIMEOUT,
                   &error_string);
    return CUDA_ERROR_LAUNCH_TIMEOUT;
  }
  *iter = all_ok ? worst_it : -worst_it;
  if (berr != nullptr) *berr = worst_berr;
  return CUDA_SUCCESS;
}

// ?POTRS: B := A^-1 B from the Cholesky factor in A (lower L or upper U = L^T).
template <typename T>
CUresult potrs_run(CULAPACKhandle h, bool upper, int n, int nrhs, const T* A, long long lda, T* B, long long ldb) {
  cudaStream_t s = h->s_panel;
  const long long rs = upper ? lda : 1, cs = upper ? 1 : lda;
  const int nblk = (n + BS - 1) / BS;
  const long long ldy = (long long)nblk * BS;
  const size_t di = round_up(sizeof(T) * (size_t)nblk * BS * BS, 256);
  CUCHOL_CHECK_CU(ensure_workspace(h, di + sizeof(T) * ldy * NR));
  T* DI = static_cast<T*>(h->ws);
  T* Y = reinterpret_cast<T*>(static_cast<char*>(h->ws) + di);
  unsigned* ctr = reinterpret_cast<unsigned*>(h->d_words + 8);   // words 8..11
  int* err = h->d_words + 3;
  CUCHOL_CHECK_CU(block_inverse<T>(A, rs, cs, n, DI, s));
  CUCHOL_CHECK_CU((trsv_attr<T, T>()));
  for (int g0 = 0; g0 < nrhs; g0 += NR) {
    const int nc = std::min(NR, nrhs - g0);
    T* Bg = B + (long long)g0 * ldb;
    CUCHOL_CHECK(cudaMemsetAsync(ctr, 0, 4 * sizeof(unsigned), s));
    trsv_fwd_kernel<T, T><<<nblk, kThreads, trsv_smem<T>(), s>>>(A, rs, cs, n, DI, Bg, ldb, nullptr, Y, ldy, nc, ctr, err,
                                                                      h->wait_limit);
    CUCHOL_CHECK(cudaGetLastError());
    trsv_bwd_kernel<T, T><<<nblk, kThreads, trsv_smem<T>(), s>>>(A, rs, cs, n, DI, Y, ldy, nullptr, Bg, ldb, Y, nc, ctr + 2,
                                                    err, h->wait_limit);
    CUCHOL_CHECK(cudaGetLastError());
    h->launches += 2;
  }
  CUCHOL_CHECK(cudaMemcpyAsync(h->h_words, h->d_words, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
  CUCHOL_CHECK(cudaStreamSynchronize(s));
  return check_engine(h);
}

}  // namespace mx
}  // namespace

// ------------------------------------------------------------------------------
// C ABI (include/cucholesky_ext.h)
// ------------------------------------------------------------------------------
namespace {
template <typename T>
CUresult api_potrs(const char* name, CULAPACKhandle h, CBlasUplo uplo, size_t n, size_t nrhs, CUdeviceptr A,
                   size_t lda, CUdeviceptr B, size_t ldb, long* info) {
  if (info == nullptr) return CUDA_ERROR_INVALID_VALUE;
  *info = 0;
  if (bad_uplo(uplo)) *info = -2;
  else if (lda < std::max<size_t>(1, n)) *info = -6;
  else if (ldb < std::max<size_t>(1, n)) *info = -8;
  if (*info != 0) {
    if (xerbla != nullptr) xerbla(name, -*info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (h == nullptr) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0 || nrhs == 0) return CUDA_SUCCESS;
  return mx::potrs_run<T>(h, uplo == CBlasUpper, (int)n, (int)nrhs, reinterpret_cast<const T*>(A), (long long)lda,
                          reinterpret_cast<T*>(B), (long long)ldb);
}
}  // namespace

extern "C" CUCHOL_EXPORT CUresult cuDpotrs(CULAPACKhandle h, CBlasUplo uplo, size_t n, size_t nrhs, CUdeviceptr A,
                                           size_t lda, CUdeviceptr B, size_t ldb, long* info) {
  return api_potrs<double>("cuDpotrs", h, uplo, n, nrhs, A, lda, B, ldb, info);
}
extern "C" CUCHOL_EXPORT CUresult cuSpotrs(CULAPACKhandle h, CBlasUplo uplo, size_t n, size_t nrhs, CUdeviceptr A,
                                           size_t lda, CUdeviceptr B, size_t ldb, long* info) {
  return api_potrs<float>("cuSpotrs", h, uplo, n, nrhs, A, lda, B, ldb, info);
}

extern "C" CUCHOL_EXPORT CUresult cuDcholMixedCreate(CUcholMixed* plan, CULAPACKhandle h, CBlasUplo uplo, size_t n,
                                                     CUdeviceptr A, size_t lda, int precision, double shift,
                                                     long* info) {
  if (plan == nullptr || info == nullptr) return CUDA_ERROR_INVALID_VALUE;
  *plan = nullptr;
  *info = 0;
  if (bad_uplo(uplo)) *info = -3;
  else if (n == 0 || n > (size_t)INT_MAX / 2) *info = -4;
  else if (lda < n) *info = -6;
  else if (precision != CUCHOL_MIXED_BF16 && precision != CUCHOL_MIXED_TF32) *info = -7;
  if (*info != 0) {
    if (xerbla != nullptr) xerbla("cuDcholMixedCreate", -*info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (h == nullptr) return CUDA_ERROR_INVALID_VALUE;
  if (precision == CUCHOL_MIXED_BF16) return mx::mixed_create<__nv_bfloat16>(plan, h, uplo, n, A, lda, shift, info);
  return mx::mixed_create<float>(plan, h, uplo, n, A, lda, shift, info);
}

// The factor's trailing-update kernel on its own: C(i, j) += alpha sum_l Q(i, l) Q(j, l)
// for i >= j, Q k-major (row i at Q + i * ldq) in BF16 or TF32 (FP32 words), C FP32
// column-major.  Queued on `stream`.
extern "C" CUCHOL_EXPORT CUresult cuSsyrkLowp(CULAPACKhandle h, int precision, size_t n, size_t k, float alpha,
                                              CUdeviceptr Q, size_t ldq, CUdeviceptr C, size_t ldc,
                                              CUstream stream) {
  long info = 0;
  const size_t esize = (precision == CUCHOL_MIXED_BF16) ? 2 : 4;
  if (precision != CUCHOL_MIXED_BF16 && precision != CUCHOL_MIXED_TF32) info = 2;
  else if (n > (size_t)INT_MAX) info = 3;
  else if (k > (size_t)INT_MAX) info = 4;
  else if (ldq < k || (ldq * esize) % 16 != 0 || (Q & 15) != 0) info = 7;
  else if (ldc < n || ldc % 4 != 0 || (C & 15) != 0) info = 9;
  if (info != 0) {
    if (xerbla != nullptr) xerbla("cuSsyrkLowp", info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (h == nullptr) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0 || k == 0) return CUDA_SUCCESS;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int* stop = h->d_words + 5;   // never set: the update has no earlier step to depend on
  CUCHOL_CHECK(cudaMemsetAsync(stop, 0, sizeof(int), s));
  if (precision == CUCHOL_MIXED_BF16)
    return mx::tc_update<__nv_bfloat16>(h, reinterpret_cast<const __nv_bfloat16*>(Q), (long long)ldq, (int)n,
                                        (int)k, 0, 0, reinterpret_cast<float*>(C), (long long)ldc, (int)n, (int)n, s,
                                        stop, alpha);
  return mx::tc_update<float>(h, reinterpret_cast<const float*>(Q), (long long)ldq, (int)n, (int)k, 0, 0,
                              reinterpret_cast<float*>(C), (long long)ldc, (int)n, (int)n, s, stop, alpha);
}

extern "C" CUCHOL_EXPORT CUresult cuDcholMixedRefactor(CUcholMixed p, long* info) {
  if (p == nullptr || info == nullptr) return CUDA_ERROR_INVALID_VALUE;
  if (p->precision == CUCHOL_MIXED_BF16) return mx::mixed_refactor<__nv_bfloat16>(p, info);
  return mx::mixed_refactor<float>(p, info);
}

extern "C" CUCHOL_EXPORT CUresult cuDcholMixedSolve(CUcholMixed p, size_t nrhs, CUdeviceptr B, size_t ldb,
                                                    CUdeviceptr X, size_t ldx, double tol, int maxit, int* iter,
                                                    double* berr) {
  if (p == nullptr || iter == nullptr || ldb < (size_t)p->n || ldx < (size_t)p->n) return CUDA_ERROR_INVALID_VALUE;
  *iter = 0;
  if (nrhs == 0) return CUDA_SUCCESS;
  return mx::mixed_solve(p, (int)nrhs, reinterpret_cast<const double*>(B), (long long)ldb,
                         reinterpret_cast<double*>(X), (long long)ldx, tol, maxit, iter, berr);
}

extern "C" CUCHOL_EXPORT CUresult cuCholMixedGetFactor(CUcholMixed p, CUdeviceptr* W, size_t* ldw, CUdeviceptr* s,
                                                       double* anorm, double* shift) {
  if (p == nullptr) return CUDA_ERROR_INVALID_VALUE;
  if (W != nullptr) *W = reinterpret_cast<CUdeviceptr>(p->W);
  if (ldw != nullptr) *ldw = (size_t)p->ldw;
  if (s != nullptr) *s = reinterpret_cast<CUdeviceptr>(p->s);
  if (anorm != nullptr) *anorm = p->anorm;
  if (shift != nullptr) *shift = p->shift;
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuCholMixedDestroy(CUcholMixed p) {
  if (p == nullptr) return CUDA_ERROR_INVALID_VALUE;
  cudaDeviceSynchronize();
  mx::free_mixed(p);
  return CUDA_SUCCESS;
}

// DSPOSV contract: iter > 0 -> refined mixed-precision solution, A unchanged;
// iter < 0 -> FP64 fallback (-3: the low-precision factor broke down, -31: no
// convergence within maxit), A holds the FP64 factor and info is cuDpotrf's.
extern "C" CUCHOL_EXPORT CUresult cuDposvMixed(CULAPACKhandle h, CBlasUplo uplo, size_t n, size_t nrhs,
                                               CUdeviceptr A, size_t lda, CUdeviceptr B, size_t ldb, CUdeviceptr X,
                                               size_t ldx, int precision, int* iter, double* berr, long* info) {
  if (iter == nullptr || info == nullptr) return CUDA_ERROR_INVALID_VALUE;
  *iter = 0;
  *info = 0;
  if (bad_uplo(uplo)) *info = -2;
  else if (lda < std::max<size_t>(1, n)) *info = -6;
  else if (ldb < std::max<size_t>(1, n)) *info = -8;
  else if (ldx < std::max<size_t>(1, n)) *info = -10;
  else if (precision != CUCHOL_MIXED_BF16 && precision != CUCHOL_MIXED_TF32) *info = -11;
  if (*info != 0) {
    if (xerbla != nullptr) xerbla("cuDposvMixed", -*info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (h == nullptr) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0 || nrhs == 0) return CUDA_SUCCESS;
  CUcholMixed p = nullptr;
  long finfo = 0;
  CUresult r = cuDcholMixedCreate(&p, h, uplo, n, A, lda, precision, -1.0, &finfo);
  if (r != CUDA_SUCCESS) return r;
  int it = 0;
  if (finfo == 0) {
    r = cuDcholMixedSolve(p, nrhs, B, ldb, X, ldx, 0.0, 0, &it, berr);
    if (r != CUDA_SUCCESS) {
      cuCholMixedDestroy(p);
      return r;
    }
  }
  cuCholMixedDestroy(p);
  if (finfo == 0 && it > 0) {
    *iter = it;
    return CUDA_SUCCESS;
  }
  *iter = (finfo != 0) ? -3 : -31;
  // FP64 fallback: X = B, factor A in place, solve
  CUCHOL_CHECK(cudaMemcpy2D(reinterpret_cast<void*>(X), ldx * sizeof(double), reinterpret_cast<const void*>(B),
                            ldb * sizeof(double), n * sizeof(double), nrhs, cudaMemcpyDeviceToDevice));
  r = cuDpotrf(h, uplo, n, A, lda, info);
  if (r != CUDA_SUCCESS || *info != 0) return r;
  long pinfo = 0;
  r = cuDpotrs(h, uplo, n, nrhs, A, lda, X, ldx, &pinfo);
  if (berr != nullptr) *berr = -1.0;
  return r;
}
