// Diagonal-block kernels: each CTA holds one jb x jb block of the logical lower
// triangle in shared memory.
//
//   potf2_block_kernel  Cholesky factor of one diagonal block (the ?POTF2 step of
//                       the blocked factor), plus optionally its inverse (used by
//                       the panel solve, which then runs as a GEMM on the tile
//                       engine) and the block's share of log det A.
//   trti2_batched_kernel  in-place inverse of every nb x nb diagonal block of a
//                       triangular matrix (the leaves of the recursive ?TRTRI).
//   diag_scan_kernel    first zero pivot of a triangular matrix in the scan order
//                       of the reference's ?trti2.
//
// The logical lower-triangle element (i, j), i >= j, lives at base[i*rs + j*cs]:
// (rs, cs) = (1, lda) for lower storage and (lda, 1) for upper storage (running the
// lower algorithm on the transposed view yields the upper factor U = L^T in place,
// without conjugation, for both real and complex types).
#pragma once
#include "scalar.cuh"

namespace cuchol {

// In-place inverse of the lower-triangular jb x jb matrix held column-major in
// shared memory S (S[i + j*LD] = L(i, j)); the strict upper part is ignored.
// Column j of inv(L), from the last column back:
//   X(j, j) = 1 / L(j, j),  X(i, j) = -X(j, j) * sum_{k=j+1..i} X(i, k) L(k, j)  (i > j)
// which is the reference's column order in lapack/dtrtri.c:70-94 (lower branch),
// with each dot product split over a group of threads.
template <typename T, int NT>
__device__ void invert_lower_smem(T* S, int LD, int jb, bool unit) {
  constexpr int G = 4;                        // threads per row
  const int tid = threadIdx.x;
  const int grp = tid / G, lane = tid % G;    // NT / G row groups
  for (int j = jb - 1; j >= 0; --j) {
    __syncthreads();
    T djj = unit ? from_real<T>(RealOf<T>(1)) : recip(S[j + j * LD]);
    // rows i = j+1 .. jb-1; the row loop runs a CTA-uniform number of times so
    // that every lane of a warp reaches the shuffles
    constexpr int RMAX = (128 + NT / G - 1) / (NT / G);   // jb <= 128
    T acc[RMAX];
    int r = 0;
    for (int base = j + 1; base < jb; base += NT / G, ++r) {
      const int i = base + grp;
      T s = zero<T>();
      if (i < jb) {
        for (int k = j + 1 + lane; k <= i; k += G) {
          T xik = (unit && k == i) ? from_real<T>(RealOf<T>(1)) : S[i + k * LD];
          mac(s, xik, S[k + j * LD]);
        }
      }
      // reduce over the G lanes of the group (adjacent lanes of one warp)
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) {
        if constexpr (Traits<T>::complex) {
          s.x += __shfl_down_sync(0xffffffffu, s.x, o, G);
          s.y += __shfl_down_sync(0xffffffffu, s.y, o, G);
        } else {
          s += __shfl_down_sync(0xffffffffu, s, o, G);
        }
      }
      if (r < RMAX) acc[r] = neg(mul(djj, s));
    }
    __syncthreads();
    r = 0;
    for (int base = j + 1; base < jb; base += NT / G, ++r) {
      const int i = base + grp;
      if (i < jb && lane == 0 && r < RMAX) S[i + j * LD] = acc[r];
    }
    if (tid == 0 && !unit) S[j + j * LD] = djj;
  }
  __syncthreads();
}

// Factor one diagonal block.  On a pivot that is <= 0 or NaN at local column k the
// block stops there (same rule as lapack/dpotrf.c:71-73), *d_info becomes
// info_base + k + 1 if it was still 0, and the partially factored block is written
// back.  With inv != nullptr (and success) inv(L) is written to inv[i + j*ldinv]
// with explicit zeros above the diagonal.  With logdet != nullptr the block adds
// 2 * sum log L(j,j) to *logdet (blocks of one matrix run in stream order, so the
// sum is deterministic).
template <typename T, int NT>
__global__ void __launch_bounds__(NT)
potf2_block_kernel(T* __restrict__ A, long long rs, long long cs, int jb,
                   T* __restrict__ inv, int ldinv, long long info_base,
                   int* __restrict__ d_info, double* __restrict__ logdet) {
  using R = RealOf<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S = reinterpret_cast<T*>(smem_raw);
  __shared__ int s_fail;
  __shared__ double s_logsum[NT / 32];
  const int LD = jb;
  const int tid = threadIdx.x;
  if (*(volatile int*)d_info != 0) return;   // an earlier block already failed

  for (int e = tid; e < jb * jb; e += NT) {
    int i = e % jb, j = e / jb;
    S[e] = (i >= j) ? A[i * rs + j * cs] : zero<T>();
  }
  if (tid == 0) s_fail = -1;

  double mylog = 0.0;
  for (int k = 0; k < jb; ++k) {
    __syncthreads();
    R d = re(S[k + k * LD]);
    if (!(d > R(0))) {                 // d <= 0 or NaN
      if (tid == 0) s_fail = k;
      break;
    }
    const R rd = R(1) / d;
    // trailing update S(i, j) -= S(i, k) conj(S(j, k)) / d,  k < j <= i < jb
    const int w = tid / 32, l = tid % 32;
    for (int j = k + 1 + w; j < jb; j += NT / 32) {
      T ljk = scale(cj(S[j + k * LD]), rd);
      for (int i = j + l; i < jb; i += 32) {
        T v = S[i + j * LD];
        mac(v, neg(S[i + k * LD]), ljk);
        S[i + j * LD] = v;
      }
    }
    __syncthreads();
    const R sd = sqrt(d);
    const R rs_ = R(1) / sd;
    for (int i = k + 1 + tid; i < jb; i += NT) S[i + k * LD] = scale(S[i + k * LD], rs_);
    if (tid == 0) {
      S[k + k * LD] = from_real<T>(sd);
      mylog += log((double)sd);
    }
  }
  __syncthreads();
  const bool failed = (s_fail >= 0);
  // write back the lower part of the block
  for (int e = tid; e < jb * jb; e += NT) {
    int i = e % jb, j = e / jb;
    if (i >= j) A[i * rs + j * cs] = S[e];
  }
  if (failed) {
    if (tid == 0) atomicCAS(d_info, 0, (int)(info_base + s_fail + 1));
    return;
  }
  if (logdet != nullptr && tid == 0) *logdet += 2.0 * mylog;
  (void)s_logsum;
  if (inv == nullptr) return;
  invert_lower_smem<T, NT>(S, LD, jb, false);
  for (int e = tid; e < jb * jb; e += NT) {
    int i = e % jb, j = e / jb;
    inv[i + (long long)j * ldinv] = (i >= j) ? S[e] : zero<T>();
  }
}

// In-place inverse of the diagonal blocks [b*nb, b*nb + jb) of a triangular matrix
// (blockIdx.x = b).  Only the lower triangle of each block is read or written;
// with unit = true the diagonal is taken as 1 and left untouched.
template <typename T, int NT>
__global__ void __launch_bounds__(NT)
trti2_batched_kernel(T* __restrict__ A, long long rs, long long cs, int n, int nb, int unit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S = reinterpret_cast<T*>(smem_raw);
  const int o = blockIdx.x * nb;
  const int jb = min(nb, n - o);
  T* B = A + o * rs + o * cs;
  for (int e = threadIdx.x; e < jb * jb; e += NT) {
    int i = e % jb, j = e / jb;
    S[e] = (i >= j) ? B[i * rs + j * cs] : zero<T>();
  }
  invert_lower_smem<T, NT>(S, jb, jb, unit != 0);
  for (int e = threadIdx.x; e < jb * jb; e += NT) {
    int i = e % jb, j = e / jb;
    if (i > j || (i == j && !unit)) B[i * rs + j * cs] = S[e];
  }
}

// Zero pivots of a non-unit triangular matrix: slot[0] = max(i+1) and
// slot[1] = min(i+1) over i with A(i,i) == 0 (slot[1] starts at INT_MAX).
template <typename T>
__global__ void diag_scan_kernel(const T* __restrict__ A, long long dstride, int n, int* __restrict__ slot) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (is_zero(A[i * dstride])) {
      atomicMax(&slot[0], i + 1);
      atomicMin(&slot[1], i + 1);
    }
  }
}

// Copy the logical-lower part of an m x n block between two views:
//   dst(i, j) = src(i, j) for i - j >= diag_off (diag_off = INT_MIN copies all).
template <typename T>
__global__ void copy_view_kernel(const T* __restrict__ src, long long s_rs, long long s_cs,
                                 T* __restrict__ dst, long long d_rs, long long d_cs,
                                 int m, int n, int lower_only, const int* __restrict__ abort_flag) {
  if (abort_flag != nullptr && *(volatile const int*)abort_flag != 0) return;
  // 32 x 8 tiles; the faster index follows the unit stride of the destination
  const bool rows_fast = (d_rs == 1);
  const int tx = threadIdx.x % 32, ty = threadIdx.x / 32;
  const int bi = blockIdx.x * 32, bj = blockIdx.y * 32;
  for (int q = ty; q < 32; q += 8) {
    int i = rows_fast ? bi + tx : bi + q;
    int j = rows_fast ? bj + q : bj + tx;
    if (i < m && j < n && (!lower_only || i >= j)) dst[i * d_rs + j * d_cs] = src[i * s_rs + j * s_cs];
  }
}

// log det from a strided diagonal: 2 * sum log(Re x[i*incx]) in double, one pass.
// Partial sums go to part[blockIdx.x]; the last CTA to finish (retirement counter,
// as in the reference's lapack/dlogdet.cu:35,93-117) adds them in index order, so
// the result is deterministic.  The counter is reset for the next call.
template <typename T, int NT>
__global__ void __launch_bounds__(NT)
logdet_kernel(const T* __restrict__ x, long long incx, long long n, double* __restrict__ part,
              unsigned int* __restrict__ counter, double* __restrict__ out) {
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT)
    s += log((double)re(x[i * incx]));
  __shared__ double red[NT / 32];
  __shared__ bool last;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < NT / 32; ++w) t += red[w];
    part[blockIdx.x] = t;
    __threadfence();
    unsigned int done = atomicAdd(counter, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t = 0.0;
    for (unsigned int b = 0; b < gridDim.x; ++b) t += ((volatile double*)part)[b];
    *out = 2.0 * t;
    *counter = 0u;
  }
}

}  // namespace cuchol
