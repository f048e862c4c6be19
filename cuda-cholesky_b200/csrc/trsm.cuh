// Row-parallel panel solve of the blocked Cholesky factorisations (?potrf and the
// mixed-precision factor): the rows below a factored diagonal block are
// independent right-hand sides of L x = b, so one CTA solves 64 of them with the
// block in shared memory, with no inverse of the block and no extra pass.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace cuchol {

__device__ __forceinline__ float round_tf32(float x) {
  uint32_t u;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(x));
  return __uint_as_float(u);
}
// Rounding of a solved panel value to a tensor-core operand type (BF16: round to
// nearest even; TF32 held in an FP32 word: round to nearest, ties away).
template <typename Op> __device__ __forceinline__ Op to_op(float x);
template <> __device__ __forceinline__ __nv_bfloat16 to_op<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <> __device__ __forceinline__ float to_op<float>(float x) { return round_tf32(x); }

// Panel solve X = B L^-T in place, row-parallel: B (m x jb, jb <= 128, logical view
// B(i, j) = B[i*brs + j*bcs]) is overwritten by X, and X also goes to out2
// (out2[i*o_rs + j*o_cs]; ROUND: rounded to the tensor-core operand type O2, BF16
// or TF32, else a plain conversion).  L: the factored jb x jb diagonal block
// (view strides lrs, lcs).  CTA: 64 rows; thread (r, cg) holds columns
// [32cg, 32cg + 32) of row r in registers.  Column block b is solved by the threads
// with cg == b (forward substitution, right-looking inside the block), published
// through shared memory, and subtracted by the threads with cg > b.  Computes in T.
template <typename T, typename TB, typename TL, typename O2, bool ROUND>
__global__ void __launch_bounds__(256, 2)
    trsm_rows_kernel(TB* __restrict__ B, long long brs, long long bcs, int m, int jb, const TL* __restrict__ L,
                     long long lrs, long long lcs, O2* __restrict__ out2, long long o_rs, long long o_cs,
                     const int* __restrict__ stop) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls = reinterpret_cast<T*>(smem_raw);   // [128][33]: L(32b + j, 32b + k)
  T* Xs = Ls + 128 * 33;                    // [64][33]: solved block
  T* rd = Xs + 64 * 33;                     // [32]: 1 / L(32b + j, 32b + j)
  if (*stop != 0) return;
  const int t = threadIdx.x, r = t & 63, cg = t >> 6;
  const int row = blockIdx.x * 64 + r;
  T x[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const int col = cg * 32 + k;
    x[k] = (row < m && col < jb) ? (T)B[(long long)row * brs + (long long)col * bcs] : T(0);
  }
  const int nblk = (jb + 31) / 32;
  for (int b = 0; b < nblk; ++b) {
    const int rows = 128 - 32 * b;   // rows of L from 32b down (zero past jb)
    __syncthreads();
    for (int e = t; e < rows * 32; e += 256) {
      const int j = e >> 5, kk = e & 31;
      const int gi = 32 * b + j, gk = 32 * b + kk;
      Ls[j * 33 + kk] = (gi < jb && gk < jb && gi >= gk) ? (T)L[(long long)gi * lrs + (long long)gk * lcs] : T(0);
    }
    __syncthreads();
    if (t < 32) rd[t] = (32 * b + t < jb) ? T(1) / Ls[t * 33 + t] : T(0);
    __syncthreads();
    if (cg == b) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        x[j] *= rd[j];
#pragma unroll
        for (int kk = j + 1; kk < 32; ++kk) x[kk] -= Ls[kk * 33 + j] * x[j];
      }
#pragma unroll
      for (int kk = 0; kk < 32; ++kk) Xs[r * 33 + kk] = x[kk];
    }
    __syncthreads();
    if (cg > b) {
      const T* Lb = Ls + (cg - b) * 32 * 33;
#pragma unroll 4
      for (int kk = 0; kk < 32; ++kk) {
        const T xk = Xs[r * 33 + kk];
#pragma unroll
        for (int j = 0; j < 32; ++j) x[j] -= Lb[j * 33 + kk] * xk;
      }
    }
  }
  if (row < m) {
#pragma unroll
    for (int k = 0; k < 32; ++k) {
      const int col = cg * 32 + k;
      if (col < jb) {
        B[(long long)row * brs + (long long)col * bcs] = (TB)x[k];
        if constexpr (ROUND) {
          out2[(long long)row * o_rs + (long long)col * o_cs] = to_op<O2>((float)x[k]);
        } else {
          out2[(long long)row * o_rs + (long long)col * o_cs] = (O2)x[k];
        }
      }
    }
  }
}

template <typename T>
constexpr size_t trsm_rows_smem() { return sizeof(T) * (128 * 33 + 64 * 33 + 32); }

}  // namespace cuchol
