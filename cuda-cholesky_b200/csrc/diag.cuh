// Small kernels of the path:
//   diag_scan_kernel    zero pivots of a triangular matrix (for the ?trtri info);
//   copy_view_kernel    copy between two strided views of a block;
//   logdet_kernel       2 * sum log(Re x[i*incx]), single pass.
//
// The logical lower-triangle element (i, j), i >= j, lives at base[i*rs + j*cs]:
// (rs, cs) = (1, lda) for lower storage and (lda, 1) for upper storage (running the
// lower algorithm on the transposed view yields the upper factor U = L^T in place,
// without conjugation, for both real and complex types).
#pragma once
#include "scalar.cuh"

namespace cuchol {

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
  if (cta_aborted(abort_flag)) return;
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
