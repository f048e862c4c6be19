// Row-parallel panel solve of the blocked Cholesky factorisations (?potrf and the
// mixed-precision factor): the rows below a factored diagonal block are
// independent right-hand sides of L x = b, so one CTA solves 64 of them with the
// block in shared memory, with no inverse of the block and no extra pass.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>
#include "scalar.cuh"

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

// Conversions between the element types the panel solve reads and writes (the
// complex types are only ever converted to themselves).
template <typename D, typename S> __device__ __forceinline__ D cvt(S x) {
  if constexpr (Traits<D>::complex) return x;
  else return (D)x;
}
// acc -= a * b
__device__ __forceinline__ void msub(float& acc, float a, float b) { acc = fmaf(-a, b, acc); }
__device__ __forceinline__ void msub(double& acc, double a, double b) { acc = fma(-a, b, acc); }
__device__ __forceinline__ void msub(cuFloatComplex& acc, cuFloatComplex a, cuFloatComplex b) {
  acc.x = fmaf(-a.x, b.x, acc.x); acc.x = fmaf(a.y, b.y, acc.x);
  acc.y = fmaf(-a.x, b.y, acc.y); acc.y = fmaf(-a.y, b.x, acc.y);
}
__device__ __forceinline__ void msub(cuDoubleComplex& acc, cuDoubleComplex a, cuDoubleComplex b) {
  acc.x = fma(-a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(-a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
}

// How the panel solve writes its second copy of X (out2, and out3 for the split).
enum : int {
  OUT_CONVERT = 0,   // out2 = X converted to O2
  OUT_ROUND = 1,     // out2 = X rounded to the tensor-core operand type O2 (BF16 or TF32)
  OUT_SPLIT = 2,     // out2 = hi = tf32(X), out3 = lo = tf32(X - hi): X = hi + lo to 2^-22
};

// Panel solve X = B L^-H in place (L^-T for real types), row-parallel: B (m x jb,
// jb <= 128, logical view B(i, j) = B[i*brs + j*bcs]) is overwritten by X, and X
// also goes to out2 (out2[i*o_rs + j*o_cs]) and, for OUT_SPLIT, out3 (same strides),
// as MODE says.  L: the factored jb x jb
// diagonal block (view strides lrs, lcs).  Each row x of X solves x L^H = b:
//   x_k = (b_k - sum_{j<k} x_j conj(L(k, j))) / L(k, k),
// so the block is staged as conj(L).  CTA: 64 rows; thread (r, cg) holds columns
// [32cg, 32cg + 32) of row r in registers.  Column block b is solved by the threads
// with cg == b (forward substitution, right-looking inside the block), published
// through shared memory, and subtracted by the threads with cg > b.  Computes in T.
// Complex double rows need up to 255 registers: one CTA per SM for that type.
template <typename T, typename TB, typename TL, typename O2, int MODE>
__global__ void __launch_bounds__(256, sizeof(T) == 16 ? 1 : 2)
    trsm_rows_kernel(TB* __restrict__ B, long long brs, long long bcs, int m, int jb, const TL* __restrict__ L,
                     long long lrs, long long lcs, O2* __restrict__ out2, long long o_rs, long long o_cs,
                     const int* __restrict__ stop, O2* __restrict__ out3) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Ls = reinterpret_cast<T*>(smem_raw);   // [128][33]: conj L(32b + j, 32b + k)
  T* Xs = Ls + 128 * 33;                    // [64][33]: solved block
  T* rd = Xs + 64 * 33;                     // [32]: 1 / L(32b + j, 32b + j)
  if (cta_aborted(stop)) return;
  const int t = threadIdx.x, r = t & 63, cg = t >> 6;
  const int row = blockIdx.x * 64 + r;
  T x[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const int col = cg * 32 + k;
    x[k] = (row < m && col < jb) ? cvt<T>(B[(long long)row * brs + (long long)col * bcs]) : zero<T>();
  }
  const int nblk = (jb + 31) / 32;
  for (int b = 0; b < nblk; ++b) {
    const int rows = 128 - 32 * b;   // rows of L from 32b down (zero past jb)
    __syncthreads();
    for (int e = t; e < rows * 32; e += 256) {
      const int j = e >> 5, kk = e & 31;
      const int gi = 32 * b + j, gk = 32 * b + kk;
      Ls[j * 33 + kk] =
          (gi < jb && gk < jb && gi >= gk) ? cj(cvt<T>(L[(long long)gi * lrs + (long long)gk * lcs])) : zero<T>();
    }
    __syncthreads();
    if (t < 32) rd[t] = (32 * b + t < jb) ? recip(Ls[t * 33 + t]) : zero<T>();
    __syncthreads();
    if (cg == b) {
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        x[j] = mul(x[j], rd[j]);
#pragma unroll
        for (int kk = j + 1; kk < 32; ++kk) msub(x[kk], Ls[kk * 33 + j], x[j]);
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
        for (int j = 0; j < 32; ++j) msub(x[j], Lb[j * 33 + kk], xk);
      }
    }
  }
  // the solved 64-row tile, staged in shared memory (the L / X buffers are idle now),
  // goes to each output in the order that is contiguous in that output
  __syncthreads();
  T* Xt = reinterpret_cast<T*>(smem_raw);   // [64][129]: Xt[r * 129 + col]
#pragma unroll
  for (int k = 0; k < 32; ++k) Xt[r * 129 + cg * 32 + k] = x[k];
  __syncthreads();
  const int rows = min(64, m - (int)blockIdx.x * 64);
  const long long row0 = (long long)blockIdx.x * 64;
  auto put = [&](auto* out, long long rs_, long long cs_, auto conv) {
    if (rs_ == 1) {        // rows contiguous: consecutive threads take consecutive rows
      for (int e = t; e < 64 * jb; e += 256) {
        const int rr = e & 63, c = e >> 6;
        if (rr < rows) out[(row0 + rr) * rs_ + (long long)c * cs_] = conv(Xt[rr * 129 + c]);
      }
    } else {               // columns contiguous (or neither): consecutive threads take consecutive columns
      for (int e = t; e < rows * jb; e += 256) {
        const int rr = e / jb, c = e - rr * jb;
        out[(row0 + rr) * rs_ + (long long)c * cs_] = conv(Xt[rr * 129 + c]);
      }
    }
  };
  put(B, brs, bcs, [](T v) { return cvt<TB>(v); });
  if constexpr (MODE == OUT_ROUND) {
    put(out2, o_rs, o_cs, [](T v) { return to_op<O2>((float)v); });
  } else if constexpr (MODE == OUT_SPLIT) {
    put(out2, o_rs, o_cs, [](T v) { return round_tf32((float)v); });
    put(out3, o_rs, o_cs, [](T v) {
      const float hi = round_tf32((float)v);
      return round_tf32((float)v - hi);
    });
  } else {
    put(out2, o_rs, o_cs, [](T v) { return cvt<O2>(v); });
  }
}

// Shared memory of trsm_rows_kernel: the diagonal block rows, the published solved
// block and the reciprocal pivots, and later the 64 x 128 output tile (padded).
template <typename T>
constexpr size_t trsm_rows_smem() {
  return sizeof(T) * ((128 * 33 + 64 * 33 + 32) > 64 * 129 ? (128 * 33 + 64 * 33 + 32) : 64 * 129);
}

}  // namespace cuchol
