// Scalar traits for the four element types of the path (s, d, c, z).
#pragma once
#include <cuComplex.h>
#include <cuda_runtime.h>

namespace cuchol {

template <typename T> struct Traits;

template <> struct Traits<float> {
  using R = float;
  static constexpr bool complex = false;
  static constexpr char prefix = 's';
};
template <> struct Traits<double> {
  using R = double;
  static constexpr bool complex = false;
  static constexpr char prefix = 'd';
};
template <> struct Traits<cuFloatComplex> {
  using R = float;
  static constexpr bool complex = true;
  static constexpr char prefix = 'c';
};
template <> struct Traits<cuDoubleComplex> {
  using R = double;
  static constexpr bool complex = true;
  static constexpr char prefix = 'z';
};

template <typename T> using RealOf = typename Traits<T>::R;

// ---- real ----
__host__ __device__ __forceinline__ float  re(float x)  { return x; }
__host__ __device__ __forceinline__ double re(double x) { return x; }
__host__ __device__ __forceinline__ float  re(cuFloatComplex x)  { return x.x; }
__host__ __device__ __forceinline__ double re(cuDoubleComplex x) { return x.x; }

__host__ __device__ __forceinline__ float  cj(float x)  { return x; }
__host__ __device__ __forceinline__ double cj(double x) { return x; }
__host__ __device__ __forceinline__ cuFloatComplex  cj(cuFloatComplex x)  { return make_cuFloatComplex(x.x, -x.y); }
__host__ __device__ __forceinline__ cuDoubleComplex cj(cuDoubleComplex x) { return make_cuDoubleComplex(x.x, -x.y); }

template <typename T> __host__ __device__ __forceinline__ T zero();
template <> __host__ __device__ __forceinline__ float  zero<float>()  { return 0.f; }
template <> __host__ __device__ __forceinline__ double zero<double>() { return 0.0; }
template <> __host__ __device__ __forceinline__ cuFloatComplex  zero<cuFloatComplex>()  { return make_cuFloatComplex(0.f, 0.f); }
template <> __host__ __device__ __forceinline__ cuDoubleComplex zero<cuDoubleComplex>() { return make_cuDoubleComplex(0.0, 0.0); }

template <typename T> __host__ __device__ __forceinline__ T from_real(RealOf<T> r);
template <> __host__ __device__ __forceinline__ float  from_real<float>(float r)   { return r; }
template <> __host__ __device__ __forceinline__ double from_real<double>(double r) { return r; }
template <> __host__ __device__ __forceinline__ cuFloatComplex  from_real<cuFloatComplex>(float r)   { return make_cuFloatComplex(r, 0.f); }
template <> __host__ __device__ __forceinline__ cuDoubleComplex from_real<cuDoubleComplex>(double r) { return make_cuDoubleComplex(r, 0.0); }

// a + b, a - b, a * b, a * s (s real)
__host__ __device__ __forceinline__ float  add(float a, float b)   { return a + b; }
__host__ __device__ __forceinline__ double add(double a, double b) { return a + b; }
__host__ __device__ __forceinline__ cuFloatComplex  add(cuFloatComplex a, cuFloatComplex b)   { return make_cuFloatComplex(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cuDoubleComplex add(cuDoubleComplex a, cuDoubleComplex b) { return make_cuDoubleComplex(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float  sub(float a, float b)   { return a - b; }
__host__ __device__ __forceinline__ double sub(double a, double b) { return a - b; }
__host__ __device__ __forceinline__ cuFloatComplex  sub(cuFloatComplex a, cuFloatComplex b)   { return make_cuFloatComplex(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cuDoubleComplex sub(cuDoubleComplex a, cuDoubleComplex b) { return make_cuDoubleComplex(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float  mul(float a, float b)   { return a * b; }
__host__ __device__ __forceinline__ double mul(double a, double b) { return a * b; }
__host__ __device__ __forceinline__ cuFloatComplex mul(cuFloatComplex a, cuFloatComplex b) {
  return make_cuFloatComplex(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cuDoubleComplex mul(cuDoubleComplex a, cuDoubleComplex b) {
  return make_cuDoubleComplex(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float  scale(float a, float s)   { return a * s; }
__host__ __device__ __forceinline__ double scale(double a, double s) { return a * s; }
__host__ __device__ __forceinline__ cuFloatComplex  scale(cuFloatComplex a, float s)   { return make_cuFloatComplex(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ cuDoubleComplex scale(cuDoubleComplex a, double s) { return make_cuDoubleComplex(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float  neg(float a)  { return -a; }
__host__ __device__ __forceinline__ double neg(double a) { return -a; }
__host__ __device__ __forceinline__ cuFloatComplex  neg(cuFloatComplex a)  { return make_cuFloatComplex(-a.x, -a.y); }
__host__ __device__ __forceinline__ cuDoubleComplex neg(cuDoubleComplex a) { return make_cuDoubleComplex(-a.x, -a.y); }

// acc += a * b  (fused where the hardware has it)
__device__ __forceinline__ void mac(float &acc, float a, float b)    { acc = fmaf(a, b, acc); }
__device__ __forceinline__ void mac(double &acc, double a, double b) { acc = fma(a, b, acc); }
__device__ __forceinline__ void mac(cuFloatComplex &acc, cuFloatComplex a, cuFloatComplex b) {
  acc.x = fmaf(a.x, b.x, acc.x); acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y); acc.y = fmaf(a.y, b.x, acc.y);
}
__device__ __forceinline__ void mac(cuDoubleComplex &acc, cuDoubleComplex a, cuDoubleComplex b) {
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
}

__host__ __device__ __forceinline__ bool is_zero(float a)  { return a == 0.f; }
__host__ __device__ __forceinline__ bool is_zero(double a) { return a == 0.0; }
__host__ __device__ __forceinline__ bool is_zero(cuFloatComplex a)  { return a.x == 0.f && a.y == 0.f; }
__host__ __device__ __forceinline__ bool is_zero(cuDoubleComplex a) { return a.x == 0.0 && a.y == 0.0; }

// 1 / a, using the standard division of the type (complex: Smith-free formula is
// enough for the well-scaled triangular pivots this path inverts)
__device__ __forceinline__ float  recip(float a)  { return 1.f / a; }
__device__ __forceinline__ double recip(double a) { return 1.0 / a; }
__device__ __forceinline__ cuFloatComplex  recip(cuFloatComplex a)  { return cuCdivf(make_cuFloatComplex(1.f, 0.f), a); }
__device__ __forceinline__ cuDoubleComplex recip(cuDoubleComplex a) { return cuCdiv(make_cuDoubleComplex(1.0, 0.0), a); }

template <typename T> __device__ __forceinline__ T conj_if(T x, bool c) { return c ? cj(x) : x; }

// CTA-uniform test of up to two abort words (the device info word of a
// factorization, a per-problem stop word).  Thread 0 reads them once and the CTA
// decides together: a word that a kernel on another stream sets while this CTA is
// starting must not split it into threads that run and threads that exit, which
// would leave the running ones waiting for the exited ones.  Every thread of the CTA
// must call it, before any other barrier.
__device__ __forceinline__ bool cta_aborted(const int* a, const int* b = nullptr) {
  __shared__ int s_abort_word;
  if (threadIdx.x == 0)
    s_abort_word = (a != nullptr && *(volatile const int*)a != 0) || (b != nullptr && *(volatile const int*)b != 0);
  __syncthreads();
  return s_abort_word != 0;
}

// Nanoseconds of the GPU's global timer (for waits bounded in time).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

}  // namespace cuchol
