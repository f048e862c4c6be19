// cuDlogdetNoAlloc: the log-determinant reduction of cuDlogdet for callers that
// cannot allocate device memory (see include/cucholesky_ext.h for who they are).
//
// The reduction needs scratch memory (one partial sum per CTA, a retirement
// counter and the result word).  cuDlogdet keeps it in its handle, which
// cuLAPACKCreate allocates; the reference's cuDlogdet even calls cuMemAlloc and
// cuMemFree on every call (lapack/dlogdet.c:56-71).  Here the scratch is a
// file-scope __device__ array instead: every GPU that loads this library holds it
// (32 KB and a few words) until the process exits, and no call allocates.
#include <cuda_runtime.h>
#include <mutex>

#include "handle.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr long long kChunk = (long long)kThreads * kPerThread;   // elements per CTA
constexpr int kMaxChunks = 4096;                                 // one partial per CTA
constexpr long long kMaxN = kChunk * kMaxChunks;                 // 8,388,608 elements

struct Scratch {
  double partial[kMaxChunks];   // 32 KB
  unsigned int counter;         // CTAs done; must be 0 when a call starts
  double result;
};

// The scratch.  In host code this name is only a stand-in for the device
// object: its device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) Scratch g_scratch;

// CTA b sums log(x[i*incx]) over its chunk [b*kChunk, (b+1)*kChunk); the last CTA
// to finish (retirement counter) adds the partials in index order, writes
// 2 * sum into sc->result and resets the counter.
__global__ void __launch_bounds__(kThreads)
logdet_static_kernel(const double* __restrict__ x, long long incx, long long n, Scratch* sc) {
  const long long base = (long long)blockIdx.x * kChunk;
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    const long long i = base + (long long)q * kThreads + threadIdx.x;
    if (i < n) s += log(x[i * incx]);
  }
  __shared__ double red[kThreads / 32];
  __shared__ bool last;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (threadIdx.x % 32 == 0) red[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) t += red[w];
    sc->partial[blockIdx.x] = t;
    __threadfence();
    last = (atomicAdd(&sc->counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double t = 0.0;
    for (unsigned int b = 0; b < gridDim.x; ++b) t += ((volatile double*)sc->partial)[b];
    sc->result = 2.0 * t;
    sc->counter = 0u;
  }
}

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
Scratch* g_addr[kMaxDevices] = {};
CUcontext g_ctx[kMaxDevices] = {};   // the context each cached address belongs to

using CtxGetCurrentFn = CUresult (*)(CUcontext*);

// The driver's cuCtxGetCurrent (this library links only the CUDA runtime).
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

// Device address of g_scratch on the current device, looked up (with that device
// current) on the first call for the device and cached together with the device's
// context: a context created since (after cudaDeviceReset the module is loaded
// again and the array may sit elsewhere) triggers a fresh lookup.
CUresult scratch_address(Scratch** out) {
  int dev = 0;
  CUCHOL_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return CUDA_ERROR_INVALID_DEVICE;
  CtxGetCurrentFn get = ctx_get_current();
  if (get == nullptr) return CUDA_ERROR_NOT_FOUND;
  CUcontext ctx = nullptr;   // null before the runtime has made a context current
  CUresult rc = get(&ctx);
  if (rc != CUDA_SUCCESS) return rc;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (ctx == nullptr || g_addr[dev] == nullptr || g_ctx[dev] != ctx) {
    void* p = nullptr;
    CUCHOL_CHECK(cudaGetSymbolAddress(&p, g_scratch));   // makes the device's context current
    if ((rc = get(&ctx)) != CUDA_SUCCESS) return rc;
    g_addr[dev] = static_cast<Scratch*>(p);
    g_ctx[dev] = ctx;
  }
  *out = g_addr[dev];
  return CUDA_SUCCESS;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) CUresult
cuDlogdetNoAlloc(CUdeviceptr x, size_t incx, size_t n, double* result, CUstream stream) {
  if (result == nullptr) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0) {
    *result = 0.0;
    return CUDA_SUCCESS;
  }
  if (n > (size_t)kMaxN) {
    // the static scratch holds one partial sum per 2048 elements
    if (xerbla != nullptr) xerbla("cuDlogdetNoAlloc", 3);
    return CUDA_ERROR_INVALID_VALUE;
  }
  Scratch* sc = nullptr;
  CUCHOL_CHECK_CU(scratch_address(&sc));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  CUCHOL_CHECK(cudaMemsetAsync(&sc->counter, 0, sizeof(unsigned int), s));
  const unsigned int grid = (unsigned int)((n + kChunk - 1) / kChunk);
  logdet_static_kernel<<<grid, kThreads, 0, s>>>(reinterpret_cast<const double*>(x), (long long)incx,
                                                  (long long)n, sc);
  CUCHOL_CHECK(cudaGetLastError());
  CUCHOL_CHECK(cudaMemcpyAsync(result, &sc->result, sizeof(double), cudaMemcpyDeviceToHost, s));
  return CUDA_SUCCESS;
}
