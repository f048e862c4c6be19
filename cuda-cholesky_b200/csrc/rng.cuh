// Counter-based GPU RNG behind the reference's cuRng32 / cuRng64 API
// (include/curng.h; reference include/rng.h:238-413), and the device SPD
// test-matrix generator cu?latmc (include/cucholesky_ext.h) built on it.
//
// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC 2011): ten rounds of two 32 x 32
// -> 64-bit products with the published multipliers and key increments; every
// 128-bit block of the stream is an independent function of (key, counter), so a
// fill is a grid-stride loop over blocks with no shared state.
//
// cu?latmc follows the reference's test generator (test/lapack/util/dlatmc.c:11-70,
// zlatmc.c): D = diag(1, c, d_2, .., d_{n-1}) with d_j uniform in [1, c], a random u,
// and A = H D H for the Householder reflection H = I - t u u^H, t = 2 / u^H u,
// expanded as A = D - u w^H - w u^H with w = t D u - s u, s = t^2 (u^H D u) / 2.  So
// A is Hermitian positive definite with eigenvalues exactly D's and condition number
// c.  Draws (the generator's [0,1] conversion, in order): d_2 .. d_{n-1}, then u
// (complex: real and imaginary part of each element in turn).
#pragma once

struct __curng32_type_st { int id; };
struct __curng64_type_st { int id; };
struct __curng32_st { uint32_t k0, k1; unsigned long long block; int sms; };
struct __curng64_st { uint32_t k0, k1; unsigned long long block; int sms; };

namespace {

__curng32_type_st k_philox32{1};
__curng64_type_st k_philox64{1};

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

__device__ __forceinline__ uint4 philox_block(unsigned long long b, uint32_t k0, uint32_t k1) {
  return philox4x32_10(make_uint4((uint32_t)b, (uint32_t)(b >> 32), 0u, 0u), k0, k1);
}

enum RngKind { RNG_RAW = 0, RNG_OO = 1, RNG_OC = 2, RNG_CO = 3, RNG_CC = 4 };

template <int KIND>
__device__ __forceinline__ float word_to_float(uint32_t w) {
  if (KIND == RNG_OO) return ((float)(w >> 9) + 0.5f) * 0x1p-23f;
  if (KIND == RNG_OC) return (float)((w >> 8) + 1u) * 0x1p-24f;
  if (KIND == RNG_CO) return (float)(w >> 8) * 0x1p-24f;
  return (float)(w >> 8) / 16777215.0f;
}

template <int KIND>
__device__ __forceinline__ double u64_to_double(unsigned long long x) {
  if (KIND == RNG_OO) return ((double)(x >> 12) + 0.5) * 0x1p-52;
  if (KIND == RNG_OC) return (double)((x >> 11) + 1ull) * 0x1p-53;
  if (KIND == RNG_CO) return (double)(x >> 11) * 0x1p-53;
  return (double)(x >> 11) / 9007199254740991.0;
}

// n 32-bit words (RNG_RAW) or floats of the stream from block block0.
template <int KIND>
__global__ void __launch_bounds__(256) rng32_kernel(uint32_t k0, uint32_t k1, unsigned long long block0, void* out,
                                                    size_t n) {
  const size_t nb = (n + 3) / 4;
  for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < nb; b += (size_t)gridDim.x * blockDim.x) {
    const uint4 w = philox_block(block0 + b, k0, k1);
    const uint32_t v[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const size_t i = 4 * b + q;
      if (i >= n) break;
      if (KIND == RNG_RAW) static_cast<uint32_t*>(out)[i] = v[q];
      else static_cast<float*>(out)[i] = word_to_float<KIND>(v[q]);
    }
  }
}

// n 64-bit integers (RNG_RAW) or doubles: two per block, low word first.
template <int KIND>
__global__ void __launch_bounds__(256) rng64_kernel(uint32_t k0, uint32_t k1, unsigned long long block0, void* out,
                                                    size_t n) {
  const size_t nb = (n + 1) / 2;
  for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < nb; b += (size_t)gridDim.x * blockDim.x) {
    const uint4 w = philox_block(block0 + b, k0, k1);
    const unsigned long long v[2] = {(unsigned long long)w.x | ((unsigned long long)w.y << 32),
                                     (unsigned long long)w.z | ((unsigned long long)w.w << 32)};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const size_t i = 2 * b + q;
      if (i >= n) break;
      if (KIND == RNG_RAW) static_cast<unsigned long long*>(out)[i] = v[q];
      else static_cast<double*>(out)[i] = u64_to_double<KIND>(v[q]);
    }
  }
}

int grid_for(size_t blocks, int sms) {
  const size_t g = (blocks + 255) / 256;
  return (int)std::max<size_t>(1, std::min<size_t>(g, (size_t)sms * 8));
}

template <typename G>
CUresult rng_sms(G g) {
  int dev = 0;
  CUCHOL_CHECK(cudaGetDevice(&dev));
  CUCHOL_CHECK(cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, dev));
  return CUDA_SUCCESS;
}

template <int KIND>
CUresult fill32(CUrng32 g, void* x, size_t n, cudaStream_t s) {
  if (g == nullptr || (x == nullptr && n > 0)) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0) return CUDA_SUCCESS;
  const size_t blocks = (n + 3) / 4;
  rng32_kernel<KIND><<<grid_for(blocks, g->sms), 256, 0, s>>>(g->k0, g->k1, g->block, x, n);
  CUCHOL_CHECK(cudaGetLastError());
  g->block += blocks;
  return CUDA_SUCCESS;
}

template <int KIND>
CUresult fill64(CUrng64 g, void* x, size_t n, cudaStream_t s) {
  if (g == nullptr || (x == nullptr && n > 0)) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0) return CUDA_SUCCESS;
  const size_t blocks = (n + 1) / 2;
  rng64_kernel<KIND><<<grid_for(blocks, g->sms), 256, 0, s>>>(g->k0, g->k1, g->block, x, n);
  CUCHOL_CHECK(cudaGetLastError());
  g->block += blocks;
  return CUDA_SUCCESS;
}

// ---- cu?latmc -------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T make_t(RealOf<T> re, RealOf<T> im);
template <> __device__ __forceinline__ cuFloatComplex make_t<cuFloatComplex>(float re, float im) {
  return make_cuFloatComplex(re, im);
}
template <> __device__ __forceinline__ cuDoubleComplex make_t<cuDoubleComplex>(double re, double im) {
  return make_cuDoubleComplex(re, im);
}

// One block: d, the sums u^H u and u^H D u (fixed-order tree, deterministic), then w.
// r: the draws (n - 2 diagonal values, then u); dw: d (n reals) then w (n elements).
template <typename T>
__global__ void __launch_bounds__(1024) latmc_vectors_kernel(const RealOf<T>* __restrict__ r, int n,
                                                             RealOf<T> c, RealOf<T>* __restrict__ d,
                                                             T* __restrict__ w) {
  using R = RealOf<T>;
  constexpr bool kCplx = sizeof(T) != sizeof(R);
  const R* ru = r + (n - 2);
  __shared__ double s_t[1024], s_s[1024];
  double tt = 0.0, ss = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const R dj = (j == 0) ? R(1) : (j == 1 ? c : r[j - 2] * (c - R(1)) + R(1));
    d[j] = dj;
    R uu;
    if constexpr (kCplx) uu = ru[2 * j] * ru[2 * j] + ru[2 * j + 1] * ru[2 * j + 1];
    else uu = ru[j] * ru[j];
    tt += (double)uu;
    ss += (double)dj * (double)uu;
  }
  s_t[threadIdx.x] = tt;
  s_s[threadIdx.x] = ss;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s_t[threadIdx.x] += s_t[threadIdx.x + o];
      s_s[threadIdx.x] += s_s[threadIdx.x + o];
    }
    __syncthreads();
  }
  const R t = R(2.0 / s_t[0]);
  const R s = t * t * R(s_s[0]) / R(2);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const R tdj = t * d[j];
    if constexpr (kCplx) {
      const R ur = ru[2 * j], ui = ru[2 * j + 1];
      w[j] = make_t<T>(tdj * ur - s * ur, tdj * ui - s * ui);
    } else {
      w[j] = tdj * ru[j] - s * ru[j];
    }
  }
}

template <typename T>
__device__ __forceinline__ T latmc_u(const RealOf<T>* ru, int i) {
  if constexpr (sizeof(T) != sizeof(RealOf<T>)) return make_t<T>(ru[2 * i], ru[2 * i + 1]);
  else return ru[i];
}

// A(i, j) = D(i, j) - u_i conj(w_j) - w_i conj(u_j) for i >= j on the 32 x 32 tile
// (I, J), I >= J, written there and, conjugated, to the mirror positions (j, i), so A is
// exactly Hermitian.
template <typename T>
__global__ void __launch_bounds__(256) latmc_fill_kernel(const RealOf<T>* __restrict__ r, const RealOf<T>* __restrict__ d,
                                                         const T* __restrict__ w, int n, T* __restrict__ A,
                                                         long long lda) {
  const int I = blockIdx.x, J = blockIdx.y;
  if (J > I) return;
  __shared__ T tile[32][33];
  const RealOf<T>* ru = r + (n - 2);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;    // 32 x 8 threads
  for (int yy = ty; yy < 32; yy += 8) {
    const int i = 32 * I + tx, j = 32 * J + yy;               // column j, consecutive rows i
    T a = zero<T>();
    if (i < n && j < n && i >= j) {
      const T ui = latmc_u<T>(ru, i), uj = latmc_u<T>(ru, j);
      a = neg(add(mul(ui, cj(w[j])), mul(w[i], cj(uj))));
      if (i == j) a = from_real<T>(d[i] + re(a));
      A[i + (long long)j * lda] = a;
    }
    tile[yy][tx] = a;
  }
  __syncthreads();
  for (int yy = ty; yy < 32; yy += 8) {
    const int i = 32 * J + tx, j = 32 * I + yy;               // mirror: A(i, j) = conj(A(j, i))
    if (i < n && j < n && i < j) A[i + (long long)j * lda] = cj(tile[tx][yy]);
  }
}

template <typename T, typename G>
CUresult latmc_run(const char* name, G g, size_t n, RealOf<T> c, CUdeviceptr A, size_t lda, cudaStream_t s) {
  using R = RealOf<T>;
  constexpr bool kCplx = sizeof(T) != sizeof(R);
  long pos = 0;
  if (n < 2) pos = 2;
  else if (!(c >= R(1))) pos = 3;
  else if (lda < n) pos = 5;
  if (pos != 0) {
    if (xerbla != nullptr) xerbla(name, pos);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (g == nullptr || A == 0 || n > (size_t)INT_MAX / 4) return CUDA_ERROR_INVALID_VALUE;
  const size_t draws = (n - 2) + (kCplx ? 2 : 1) * n;
  const size_t bytes = sizeof(R) * (draws + n) + sizeof(T) * n + 256;
  void* buf = nullptr;
  CUCHOL_CHECK(cudaMallocAsync(&buf, bytes, s));
  R* r = static_cast<R*>(buf);
  R* d = r + draws;
  T* w = reinterpret_cast<T*>(static_cast<char*>(buf) + ((sizeof(R) * (draws + n) + 15) & ~size_t(15)));
  CUresult rc;
  if constexpr (sizeof(R) == 4) rc = fill32<RNG_CC>(g, r, draws, s);
  else rc = fill64<RNG_CC>(g, r, draws, s);
  if (rc == CUDA_SUCCESS) {
    latmc_vectors_kernel<T><<<1, 1024, 0, s>>>(r, (int)n, c, d, w);
    rc = to_cu(cudaGetLastError());
  }
  if (rc == CUDA_SUCCESS) {
    const unsigned nt = (unsigned)((n + 31) / 32);
    latmc_fill_kernel<T><<<dim3(nt, nt), 256, 0, s>>>(r, d, w, (int)n, reinterpret_cast<T*>(A), (long long)lda);
    rc = to_cu(cudaGetLastError());
  }
  cudaError_t e = cudaFreeAsync(buf, s);
  if (rc != CUDA_SUCCESS) return rc;
  CUCHOL_CHECK(e);
  return CUDA_SUCCESS;
}

}  // namespace

extern "C" {
CUCHOL_EXPORT const CUrng32_t philox32_t = &k_philox32;
CUCHOL_EXPORT const CUrng64_t philox64_t = &k_philox64;
}

extern "C" CUCHOL_EXPORT CUresult cuRng32Create(CUrng32* g, const CUrng32_t type) {
  if (g == nullptr || type != philox32_t) return CUDA_ERROR_INVALID_VALUE;
  auto* p = new (std::nothrow) __curng32_st{0u, 0u, 0ull, 0};
  if (p == nullptr) return CUDA_ERROR_OUT_OF_MEMORY;
  CUresult r = rng_sms(p);
  if (r != CUDA_SUCCESS) {
    delete p;
    return r;
  }
  *g = p;
  return CUDA_SUCCESS;
}
extern "C" CUCHOL_EXPORT CUresult cuRng32Destroy(CUrng32 g) {
  if (g == nullptr) return CUDA_ERROR_INVALID_VALUE;
  delete g;
  return CUDA_SUCCESS;
}
extern "C" CUCHOL_EXPORT CUresult cuRng32Set(const CUrng32 g, uint32_t seed) {
  if (g == nullptr) return CUDA_ERROR_INVALID_VALUE;
  g->k0 = seed;
  g->k1 = 0u;
  g->block = 0ull;
  return CUDA_SUCCESS;
}
extern "C" CUCHOL_EXPORT CUresult cuRng32Get(const CUrng32 g, CUdeviceptr x, size_t n) {
  return fill32<RNG_RAW>(g, reinterpret_cast<void*>(x), n, 0);
}
extern "C" CUCHOL_EXPORT CUresult cuRng32GetOpenOpen(const CUrng32 g, CUdeviceptr x, size_t n) {
  return fill32<RNG_OO>(g, reinterpret_cast<void*>(x), n, 0);
}
extern "C" CUCHOL_EXPORT CUresult cuRng32GetOpenClose(const CUrng32 g, CUdeviceptr x, size_t n) {
  return fill32<RNG_OC>(g, reinterpret_cast<void*>(x), n, 0);
}
extern "C" CUCHOL_EXPORT CUresult cuRng32GetCloseOpen(const CUrng32 g, CUdeviceptr x, size_t n) {
  return fill32<RNG_CO>(g, reinterpret_cast<void*>(x), n, 0);
}
extern "C" CUCHOL_EXPORT CUresult cuRng32GetCloseClose(const CUrng32 g, CUdeviceptr x, size_t n) {
  return fill32<RNG_CC>(g, reinterpret_cast<void*>(x), n, 0);
}

extern "C" CUCHOL_EXPORT CUresult cuRng64Create(CUrng64* g, const CUrng64_t type) {
  if (g == nullptr || type != philox64_t) return CUDA_ERROR_INVALID_VALUE;
  auto* p = new (std::nothrow) __curng64_st{0u, 0u, 0ull, 0};
  if (p == nullptr) return CUDA_ERROR_OUT_OF_MEMORY;
  CUresult r = rng_sms(p);
  if (r != CUDA_SUCCESS) {
    delete p;
    return r;
  }
  *g = p;
  return CUDA_SUCCESS;
}
extern "C" CUCHOL_EXPORT CUresult cuRng64Destroy(CUrng64 g) {
  if (g == nullptr) return CUDA_ERROR_INVALID_VALUE;
  delete g;
  return CUDA_SUCCESS;
}
extern "C" CUCHOL_EXPORT CUresult cuRng64Set(const CUrng64 g, uint64_t seed) {
  if (g == nullptr) return CUDA_ERROR_INVALID_VALUE;
  g->k0 = (uint32_t)seed;
  g->k1 = (uint32_t)(seed >> 32);
  g->block = 0ull;
  return CUDA_SUCCESS;
}
extern "C" CUCHOL_EXPORT CUresult cuRng64Get(const CUrng64 g, CUdeviceptr x, size_t n) {
  return fill64<RNG_RAW>(g, reinterpret_cast<void*>(x), n, 0);
}
extern "C" CUCHOL_EXPORT CUresult cuRng64GetOpenOpen(const CUrng64 g, CUdeviceptr x, size_t n) {
  return fill64<RNG_OO>(g, reinterpret_cast<void*>(x), n, 0);
}
extern "C" CUCHOL_EXPORT CUresult cuRng64GetOpenClose(const CUrng64 g, CUdeviceptr x, size_t n) {
  return fill64<RNG_OC>(g, reinterpret_cast<void*>(x), n, 0);
}
extern "C" CUCHOL_EXPORT CUresult cuRng64GetCloseOpen(const CUrng64 g, CUdeviceptr x, size_t n) {
  return fill64<RNG_CO>(g, reinterpret_cast<void*>(x), n, 0);
}
extern "C" CUCHOL_EXPORT CUresult cuRng64GetCloseClose(const CUrng64 g, CUdeviceptr x, size_t n) {
  return fill64<RNG_CC>(g, reinterpret_cast<void*>(x), n, 0);
}

extern "C" CUCHOL_EXPORT CUresult cuSlatmc(CUrng32 g, size_t n, float c, CUdeviceptr A, size_t lda, CUstream s) {
  return latmc_run<float>("cuSlatmc", g, n, c, A, lda, reinterpret_cast<cudaStream_t>(s));
}
extern "C" CUCHOL_EXPORT CUresult cuDlatmc(CUrng64 g, size_t n, double c, CUdeviceptr A, size_t lda, CUstream s) {
  return latmc_run<double>("cuDlatmc", g, n, c, A, lda, reinterpret_cast<cudaStream_t>(s));
}
extern "C" CUCHOL_EXPORT CUresult cuClatmc(CUrng32 g, size_t n, float c, CUdeviceptr A, size_t lda, CUstream s) {
  return latmc_run<cuFloatComplex>("cuClatmc", g, n, c, A, lda, reinterpret_cast<cudaStream_t>(s));
}
extern "C" CUCHOL_EXPORT CUresult cuZlatmc(CUrng64 g, size_t n, double c, CUdeviceptr A, size_t lda, CUstream s) {
  return latmc_run<cuDoubleComplex>("cuZlatmc", g, n, c, A, lda, reinterpret_cast<cudaStream_t>(s));
}
