// Host-memory routines of include/lapack.h and the device list of
// include/cumultigpu.h (reference include/lapack.h:117-158, include/cumultigpu.h).
//
// The reference's cuMultiGPU?potrf (lapack/dpotrf.c:298-366) keeps A in host memory
// for the whole factorization: every SYRK/GEMM/TRSM of the blocked algorithm is
// tiled across the GPUs with its operand slabs staged from host memory per tile
// (blas/dgemm.c:211-430), and each diagonal block is factored on the host.  On a
// B200 one matrix of any size the reference handles fits in the GPU's 180 GB, so
// the matrix crosses the bus once each way instead:
//   1. the `uplo` triangle is copied to the GPU in 256-column blocks, each one 2-D
//      copy of the block column's trapezoid (the other triangle crosses the bus only
//      inside the diagonal blocks);
//   2. the single-GPU driver runs on the copy (potrf_run, trtri_run, lauum_run);
//   3. the triangle is copied back.
// ?potrf with page-locked (or device) memory overlaps both copies with the
// factorization.  Copy back: each block column of the factor is queued on an
// outbound copy stream behind the work that finishes it.  Copy in: the matrix is
// cut into tall panels (1024 columns wide up to the middle column, then the second
// half in one), copied in that order and factored left-looking panel by panel as
// they land:
//   * a tall panel receives the updates of the columns left of its predecessor on a
//     background stream while the predecessor is factored, then the updates of the
//     predecessor's columns, then potrf_run factors it (right-looking inside,
//     trailing updates restricted to its own columns);
//   * the last panel receives the updates of each tall panel as soon as that panel
//     is factored and the last panel has landed, on a lowest-priority stream: this
//     bulk of the work fills the SMs that the latency-bound tall-panel
//     factorizations leave idle;
//   * then potrf_run factors the last panel right-looking.
// Background updates run in launches of at most 1024 columns of K, so the panel
// stream's one-CTA kernels wait little for an SM.  Pageable memory is copied in
// before and back after the driver (a copy to pageable memory returns only when it
// is done, which would stall the queueing of the schedule).
// A call returns when its copies have landed.  The device buffer is cached in the
// handle (grow-only, leading dimension rounded up to 32 elements).
#pragma once

namespace {

struct DeviceGuard {
  int prev = -1;
  cudaError_t err;
  explicit DeviceGuard(int d) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    err = cudaSetDevice(d);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

struct __cumultigpu_st {
  std::vector<int> devices;
};

struct __cumultigpulapackhandle_st {
  int device = 0;                   // the CUmultiGPU's first device
  CULAPACKhandle h = nullptr;       // single-GPU handle on that device
  cudaStream_t s_copy = nullptr;    // host -> device copies (and all copies of the
                                    // routines that do not overlap them)
  cudaStream_t s_out = nullptr;     // device -> host copies overlapped with ?potrf
  cudaEvent_t ev = nullptr;
  cudaStream_t s_gemm = nullptr;    // ?potrf: updates of the next tall panel
  cudaStream_t s_tail = nullptr;    // ?potrf: updates of the last panel (low priority)
  cudaEvent_t ev_tail = nullptr;
  std::vector<cudaEvent_t> ev_in;   // one per tall panel copied in
  std::vector<cudaEvent_t> ev_a;    // one per tall panel: its early updates are done
  void* buf = nullptr;              // staged matrix (grow-only)
  size_t buf_bytes = 0;
  unsigned long long h2d_bytes = 0, d2h_bytes = 0;   // bytes copied, since creation
};

namespace {

constexpr size_t kStageCols = 256;   // columns per host <-> device copy

CUresult stage_buffer(CUmultiGPULAPACKhandle hh, size_t bytes) {
  if (bytes <= hh->buf_bytes) return CUDA_SUCCESS;
  if (hh->buf != nullptr) {
    CUCHOL_CHECK(cudaFree(hh->buf));
    hh->buf = nullptr;
    hh->buf_bytes = 0;
  }
  CUCHOL_CHECK(dev_malloc(&hh->buf, bytes));
  hh->buf_bytes = bytes;
  return CUDA_SUCCESS;
}

// Page-locked host memory, device memory and managed memory take asynchronous
// copies; pageable memory does not.
bool async_copyable(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// The `uplo` triangle of an n x n column-major matrix, block column by block
// column: lower, rows j .. n-1 of columns j .. j+w-1; upper, rows 0 .. j+w-1.
template <typename T>
CUresult copy_triangle(T* dst, size_t ldd, const T* src, size_t lds, size_t n, bool upper, cudaStream_t s,
                       unsigned long long* bytes) {
  for (size_t j = 0; j < n; j += kStageCols) {
    const size_t w = std::min(kStageCols, n - j);
    const size_t r0 = upper ? 0 : j, rows = upper ? j + w : n - j;
    CUCHOL_CHECK(cudaMemcpy2DAsync(dst + r0 + j * ldd, ldd * sizeof(T), src + r0 + j * lds, lds * sizeof(T),
                                   rows * sizeof(T), w, cudaMemcpyDefault, s));
    *bytes += rows * w * sizeof(T);
  }
  return CUDA_SUCCESS;
}

// Logical block columns c0 .. c1-1 of the `uplo` triangle, logical rows from each
// piece's first column down: lower, physical columns (rows j .. n-1 of columns
// j .. j+w-1); upper, physical rows (columns j .. n-1 of rows j .. j+w-1).
template <typename T>
CUresult copy_panel(T* dst, size_t ldd, const T* src, size_t lds, size_t n, bool upper, size_t c0, size_t c1,
                    cudaStream_t s, unsigned long long* bytes) {
  for (size_t j = c0; j < c1; j += kStageCols) {
    const size_t w = std::min(kStageCols, c1 - j), len = n - j;
    const size_t width = upper ? w : len, height = upper ? len : w;
    CUCHOL_CHECK(cudaMemcpy2DAsync(dst + j + j * ldd, ldd * sizeof(T), src + j + j * lds, lds * sizeof(T),
                                   width * sizeof(T), height, cudaMemcpyDefault, s));
    *bytes += len * w * sizeof(T);
  }
  return CUDA_SUCCESS;
}

// Copies the triangle in, and orders the handle's streams after the copies.
template <typename T>
CUresult stage_in(CUmultiGPULAPACKhandle hh, const T* A, size_t lda, size_t n, bool upper, T** D, size_t* ldd) {
  *ldd = round_up(n, 32);
  CUCHOL_CHECK_CU(stage_buffer(hh, sizeof(T) * *ldd * n));
  *D = static_cast<T*>(hh->buf);
  CUCHOL_CHECK_CU(copy_triangle<T>(*D, *ldd, A, lda, n, upper, hh->s_copy, &hh->h2d_bytes));
  CUCHOL_CHECK(cudaEventRecord(hh->ev, hh->s_copy));
  CUCHOL_CHECK(cudaStreamWaitEvent(hh->h->s_panel, hh->ev, 0));
  CUCHOL_CHECK(cudaStreamWaitEvent(hh->h->s_update, hh->ev, 0));
  return CUDA_SUCCESS;
}

// Ends a call: waits for the copy streams whatever happened before, and returns the
// first error.
inline CUresult finish(CUmultiGPULAPACKhandle hh, CUresult r) {
  cudaError_t e = cudaStreamSynchronize(hh->s_copy);
  cudaError_t e2 = cudaStreamSynchronize(hh->s_out);
  cudaError_t e3 = cudaStreamSynchronize(hh->s_gemm);
  cudaError_t e4 = cudaStreamSynchronize(hh->s_tail);
  if (r != CUDA_SUCCESS) return r;
  CUCHOL_CHECK(e);
  CUCHOL_CHECK(e2);
  CUCHOL_CHECK(e3);
  CUCHOL_CHECK(e4);
  return CUDA_SUCCESS;
}

constexpr size_t kPanelCols = 1024;    // tall-panel width of the streamed ?potrf

// Column boundaries of the tall panels: 1024 wide while the panel ends at or
// before the middle column, then one panel to the end.
inline std::vector<size_t> panel_plan(size_t n) {
  std::vector<size_t> b{0};
  while (b.back() + kPanelCols <= n / 2) b.push_back(b.back() + kPanelCols);
  if (b.back() < n) b.push_back(n);
  return b;
}

// Argument checks of the reference's host-memory drivers (lapack/dpotrf.c:302-308:
// only lda, at position 4; position 5 for ?trtri).
inline bool host_args(const char* name, size_t n, size_t lda, long pos, long* info) {
  *info = 0;
  if (lda < n) {
    *info = -pos;
    if (xerbla != nullptr) xerbla(name, pos);
    return false;
  }
  return true;
}

template <typename T>
CUresult host_potrf_run(CUmultiGPULAPACKhandle hh, bool upper, size_t n, T* A, size_t lda, long* info) {
  CULAPACKhandle h = hh->h;
  const size_t ldd = round_up(n, 32);
  CUCHOL_CHECK_CU(stage_buffer(hh, sizeof(T) * ldd * n));
  T* D = static_cast<T*>(hh->buf);
  const long long rs = upper ? (long long)ldd : 1, cs = upper ? 1 : (long long)ldd;
  auto at = [&](size_t i, size_t j) { return D + (long long)i * rs + (long long)j * cs; };
  if (!async_copyable(A)) {
    // pageable: copy in, factor, copy back
    CUCHOL_CHECK_CU(copy_triangle<T>(D, ldd, A, lda, n, upper, hh->s_copy, &hh->h2d_bytes));
    CUCHOL_CHECK(cudaStreamSynchronize(hh->s_copy));
    CUCHOL_CHECK_CU(potrf_run<T>(h, upper, (int)n, D, (long long)ldd, info, nullptr));
    return copy_triangle<T>(A, lda, D, ldd, n, upper, hh->s_copy, &hh->d2h_bytes);
  }
  const std::vector<size_t> plan = panel_plan(n);
  const size_t panels = plan.size() - 1;
  while (hh->ev_in.size() < panels) {
    cudaEvent_t e;
    CUCHOL_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    hh->ev_in.push_back(e);
  }
  // every copy in is queued at once, in panel order
  for (size_t r = 0; r < panels; ++r) {
    CUCHOL_CHECK_CU(copy_panel<T>(D, ldd, A, lda, n, upper, plan[r], plan[r + 1], hh->s_copy, &hh->h2d_bytes));
    CUCHOL_CHECK(cudaEventRecord(hh->ev_in[r], hh->s_copy));
  }
  while (hh->ev_a.size() < panels) {
    cudaEvent_t e;
    CUCHOL_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    hh->ev_a.push_back(e);
  }
  const T minus_one = from_real<T>(RealOf<T>(-1)), one = from_real<T>(RealOf<T>(1));
  // A(c0:, c0:c0+w) -= L(c0:, k0:k1) L(c0:c0+w, k0:k1)^H, lower-only on the panel's
  // diagonal block, in launches of at most 1024 columns of L each: a tile of a
  // background launch then holds its SM for a fraction of a millisecond, so the
  // panel stream's one-CTA kernels find a free SM soon after they are queued.
  auto catch_up = [&](size_t c0, size_t w, size_t k0, size_t k1, cudaStream_t s) -> CUresult {
    for (size_t k = k0; k < k1; k += kPanelCols) {
      GemmProblem<T> u = problem<T>();
      u.a = at(c0, k); u.a_rs = rs; u.a_ks = cs;
      u.b = at(c0, k); u.b_rs = rs; u.b_ks = cs; u.conj_b = 1;
      u.c = at(c0, c0); u.c_rs = rs; u.c_cs = cs;
      u.cin = u.c; u.cin_rs = rs; u.cin_cs = cs;
      u.alpha = minus_one; u.beta = one;
      u.lower_only = 1; u.real_diag = 1;
      u.m = (int)(n - c0); u.n = (int)w; u.k = (int)std::min(kPanelCols, k1 - k);
      CUCHOL_CHECK_CU(gemm<T>(h, u, s, nullptr));
    }
    return CUDA_SUCCESS;
  };
  // A tall panel r receives the updates of columns 0 .. plan[r-1]-1 in one GEMM on a
  // low-priority stream while panel r-1 is factored (those columns are final by
  // then), and the updates of panel r-1's columns on the panel stream after it.  The
  // last panel (the second half) takes the updates of each tall panel as soon as that
  // panel is factored and the last panel has landed, on a second low-priority stream,
  // so they fill the GPU around the latency-bound tall-panel factorizations.
  const size_t last = panels - 1;
  for (size_t r = 0; r < panels; ++r) {
    const size_t c0 = plan[r], w = plan[r + 1] - c0;
    CUCHOL_CHECK(cudaStreamWaitEvent(h->s_panel, hh->ev_in[r], 0));
    CUCHOL_CHECK(cudaStreamWaitEvent(h->s_update, hh->ev_in[r], 0));
    if (r >= 1) {
      if (r == last) {
        if (r >= 2) CUCHOL_CHECK(cudaStreamWaitEvent(h->s_panel, hh->ev_tail, 0));
      } else if (r >= 2) {
        CUCHOL_CHECK(cudaStreamWaitEvent(h->s_panel, hh->ev_a[r], 0));
      }
      CUCHOL_CHECK_CU(catch_up(c0, w, plan[r - 1], c0, h->s_panel));
    }
    if (r >= 1 && r + 1 < last) {
      CUCHOL_CHECK(cudaStreamWaitEvent(hh->s_gemm, hh->ev_in[r + 1], 0));
      CUCHOL_CHECK_CU(catch_up(plan[r + 1], plan[r + 2] - plan[r + 1], 0, c0, hh->s_gemm));
      CUCHOL_CHECK(cudaEventRecord(hh->ev_a[r + 1], hh->s_gemm));
    }
    if (r >= 1 && r < last) {
      if (r == 1) CUCHOL_CHECK(cudaStreamWaitEvent(hh->s_tail, hh->ev_in[last], 0));
      CUCHOL_CHECK_CU(catch_up(plan[last], n - plan[last], plan[r - 1], c0, hh->s_tail));
      CUCHOL_CHECK(cudaEventRecord(hh->ev_tail, hh->s_tail));
    }
    FinalColumns back = [&](int c, int jb, cudaStream_t s) -> CUresult {
      CUCHOL_CHECK(cudaEventRecord(hh->ev, s));
      CUCHOL_CHECK(cudaStreamWaitEvent(hh->s_out, hh->ev, 0));
      const size_t g = c0 + (size_t)c, rows = n - g;
      const size_t width = upper ? (size_t)jb : rows, height = upper ? rows : (size_t)jb;
      CUCHOL_CHECK(cudaMemcpy2DAsync(A + g + g * lda, lda * sizeof(T), D + g + g * ldd, ldd * sizeof(T),
                                     width * sizeof(T), height, cudaMemcpyDefault, hh->s_out));
      hh->d2h_bytes += rows * (size_t)jb * sizeof(T);
      return CUDA_SUCCESS;
    };
    long pinfo = 0;
    CUCHOL_CHECK_CU(potrf_run<T>(h, upper, (int)(n - c0), at(c0, c0), (long long)ldd, &pinfo, nullptr, &back,
                                 (int)w));
    if (pinfo != 0) {
      *info = (long)c0 + pinfo;
      return CUDA_SUCCESS;
    }
  }
  *info = 0;
  return CUDA_SUCCESS;
}

template <typename T>
CUresult host_potrf(const char* name, CUmultiGPULAPACKhandle hh, CBlasUplo uplo, size_t n, T* A, size_t lda,
                    long* info) {
  if (!host_args(name, n, lda, 4, info)) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0) return CUDA_SUCCESS;
  if (hh == nullptr || A == nullptr || bad_uplo(uplo) || n > (size_t)INT_MAX) return CUDA_ERROR_INVALID_VALUE;
  DeviceGuard g(hh->device);
  CUCHOL_CHECK(g.err);
  CUCHOL_CHECK_CU(finish(hh, host_potrf_run<T>(hh, uplo == CBlasUpper, n, A, lda, info)));
  return *info > 0 ? CUDA_ERROR_INVALID_VALUE : CUDA_SUCCESS;
}

template <typename T>
CUresult host_trtri(const char* name, CUmultiGPULAPACKhandle hh, CBlasUplo uplo, CBlasDiag diag, size_t n, T* A,
                    size_t lda, long* info) {
  if (!host_args(name, n, lda, 5, info)) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0) return CUDA_SUCCESS;
  if (hh == nullptr || A == nullptr || bad_uplo(uplo) || n > (size_t)INT_MAX) return CUDA_ERROR_INVALID_VALUE;
  DeviceGuard g(hh->device);
  CUCHOL_CHECK(g.err);
  const bool upper = (uplo == CBlasUpper);
  T* D;
  size_t ldd;
  CUresult r = stage_in<T>(hh, A, lda, n, upper, &D, &ldd);
  if (r == CUDA_SUCCESS) r = trtri_run<T>(hh->h, upper, diag == CBlasUnit, (int)n, D, (long long)ldd, info);
  // a singular matrix is left unmodified: nothing to copy back
  if (r == CUDA_SUCCESS && *info == 0)
    r = copy_triangle<T>(A, lda, D, ldd, n, upper, hh->s_copy, &hh->d2h_bytes);
  CUCHOL_CHECK_CU(finish(hh, r));
  return *info > 0 ? CUDA_ERROR_INVALID_VALUE : CUDA_SUCCESS;
}

template <typename T>
CUresult host_lauum(const char* name, CUmultiGPULAPACKhandle hh, CBlasUplo uplo, size_t n, T* A, size_t lda,
                    long* info) {
  if (!host_args(name, n, lda, 4, info)) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0) return CUDA_SUCCESS;
  if (hh == nullptr || A == nullptr || bad_uplo(uplo) || n > (size_t)INT_MAX) return CUDA_ERROR_INVALID_VALUE;
  DeviceGuard g(hh->device);
  CUCHOL_CHECK(g.err);
  const bool upper = (uplo == CBlasUpper);
  T* D;
  size_t ldd;
  CUresult r = stage_in<T>(hh, A, lda, n, upper, &D, &ldd);
  if (r == CUDA_SUCCESS) r = lauum_run<T>(hh->h, upper, (int)n, D, (long long)ldd);
  if (r == CUDA_SUCCESS) r = copy_triangle<T>(A, lda, D, ldd, n, upper, hh->s_copy, &hh->d2h_bytes);
  return finish(hh, r);
}

template <typename T>
CUresult host_potri(const char* name, CUmultiGPULAPACKhandle hh, CBlasUplo uplo, size_t n, T* A, size_t lda,
                    long* info) {
  if (!host_args(name, n, lda, 4, info)) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0) return CUDA_SUCCESS;
  if (hh == nullptr || A == nullptr || bad_uplo(uplo) || n > (size_t)INT_MAX) return CUDA_ERROR_INVALID_VALUE;
  DeviceGuard g(hh->device);
  CUCHOL_CHECK(g.err);
  const bool upper = (uplo == CBlasUpper);
  T* D;
  size_t ldd;
  CUresult r = stage_in<T>(hh, A, lda, n, upper, &D, &ldd);
  if (r == CUDA_SUCCESS) r = trtri_run<T>(hh->h, upper, false, (int)n, D, (long long)ldd, info);
  if (r == CUDA_SUCCESS && *info == 0) r = lauum_run<T>(hh->h, upper, (int)n, D, (long long)ldd);
  if (r == CUDA_SUCCESS && *info == 0)
    r = copy_triangle<T>(A, lda, D, ldd, n, upper, hh->s_copy, &hh->d2h_bytes);
  CUCHOL_CHECK_CU(finish(hh, r));
  return *info > 0 ? CUDA_ERROR_INVALID_VALUE : CUDA_SUCCESS;
}

}  // namespace

// ---- device list (reference include/cumultigpu.h:61-97) --------------------------
extern "C" CUCHOL_EXPORT CUresult cuMultiGPUCreate(CUmultiGPU* mgpu, CUdevice* devices, int n) {
  if (mgpu == nullptr || devices == nullptr || n < 1) return CUDA_ERROR_INVALID_VALUE;
  int count = 0;
  CUCHOL_CHECK(cudaGetDeviceCount(&count));
  for (int i = 0; i < n; ++i)
    if (devices[i] < 0 || devices[i] >= count) return CUDA_ERROR_INVALID_DEVICE;
  auto* m = new (std::nothrow) __cumultigpu_st;
  if (m == nullptr) return CUDA_ERROR_OUT_OF_MEMORY;
  m->devices.assign(devices, devices + n);
  *mgpu = m;
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuMultiGPUDestroy(CUmultiGPU mgpu) {
  if (mgpu == nullptr) return CUDA_ERROR_INVALID_VALUE;
  delete mgpu;
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT int cuMultiGPUGetContextCount(CUmultiGPU mgpu) {
  return mgpu == nullptr ? 0 : (int)mgpu->devices.size();
}

extern "C" CUCHOL_EXPORT CUresult cuMultiGPUSynchronize(CUmultiGPU mgpu) {
  if (mgpu == nullptr) return CUDA_ERROR_INVALID_VALUE;
  for (int d : mgpu->devices) {
    DeviceGuard g(d);
    CUCHOL_CHECK(g.err);
    CUCHOL_CHECK(cudaDeviceSynchronize());
  }
  return CUDA_SUCCESS;
}

// ---- host-memory LAPACK handle (reference include/lapack.h:119-122, lapack/handle.c:90-108)
extern "C" CUCHOL_EXPORT CUresult cuMultiGPULAPACKCreate(CUmultiGPULAPACKhandle* handle, CUmultiGPU mgpu) {
  if (handle == nullptr || mgpu == nullptr || mgpu->devices.empty()) return CUDA_ERROR_INVALID_VALUE;
  auto* hh = new (std::nothrow) __cumultigpulapackhandle_st();
  if (hh == nullptr) return CUDA_ERROR_OUT_OF_MEMORY;
  hh->device = mgpu->devices[0];
  DeviceGuard g(hh->device);
  CUresult r = (g.err == cudaSuccess) ? cuLAPACKCreate(&hh->h) : to_cu(g.err);
  if (r == CUDA_SUCCESS) r = to_cu(cudaStreamCreateWithFlags(&hh->s_copy, cudaStreamNonBlocking));
  if (r == CUDA_SUCCESS) r = to_cu(cudaStreamCreateWithFlags(&hh->s_out, cudaStreamNonBlocking));
  int lo = 0, hi = 0;
  if (r == CUDA_SUCCESS) r = to_cu(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  // the next panel's updates (on the panel chain) rank with the factorization's own
  // trailing updates; the last panel's updates only fill SMs left idle
  const int mid = (hi < lo - 1) ? (lo + hi) / 2 : lo;
  if (r == CUDA_SUCCESS) r = to_cu(cudaStreamCreateWithPriority(&hh->s_gemm, cudaStreamNonBlocking, mid));
  if (r == CUDA_SUCCESS) r = to_cu(cudaStreamCreateWithPriority(&hh->s_tail, cudaStreamNonBlocking, lo));
  if (r == CUDA_SUCCESS) r = to_cu(cudaEventCreateWithFlags(&hh->ev_tail, cudaEventDisableTiming));
  if (r == CUDA_SUCCESS) r = to_cu(cudaEventCreateWithFlags(&hh->ev, cudaEventDisableTiming));
  if (r != CUDA_SUCCESS) {
    if (hh->ev) cudaEventDestroy(hh->ev);
    if (hh->s_out) cudaStreamDestroy(hh->s_out);
    if (hh->ev_tail) cudaEventDestroy(hh->ev_tail);
    if (hh->s_tail) cudaStreamDestroy(hh->s_tail);
    if (hh->s_gemm) cudaStreamDestroy(hh->s_gemm);
    if (hh->s_copy) cudaStreamDestroy(hh->s_copy);
    if (hh->h) cuLAPACKDestroy(hh->h);
    delete hh;
    return r;
  }
  *handle = hh;
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuMultiGPULAPACKDestroy(CUmultiGPULAPACKhandle hh) {
  if (hh == nullptr) return CUDA_ERROR_INVALID_VALUE;
  DeviceGuard g(hh->device);
  CUCHOL_CHECK(g.err);
  CUCHOL_CHECK(cudaStreamSynchronize(hh->s_copy));
  CUCHOL_CHECK(cudaStreamSynchronize(hh->s_out));
  CUCHOL_CHECK(cudaStreamSynchronize(hh->s_gemm));
  CUCHOL_CHECK(cudaStreamSynchronize(hh->s_tail));
  if (hh->buf) cudaFree(hh->buf);
  cudaEventDestroy(hh->ev);
  cudaEventDestroy(hh->ev_tail);
  cudaStreamDestroy(hh->s_tail);
  for (cudaEvent_t e : hh->ev_in) cudaEventDestroy(e);
  for (cudaEvent_t e : hh->ev_a) cudaEventDestroy(e);
  cudaStreamDestroy(hh->s_gemm);
  cudaStreamDestroy(hh->s_out);
  cudaStreamDestroy(hh->s_copy);
  CUresult r = cuLAPACKDestroy(hh->h);
  delete hh;
  return r;
}

extern "C" CUCHOL_EXPORT CUresult cuMultiGPULAPACKSynchronize(CUmultiGPULAPACKhandle hh) {
  if (hh == nullptr) return CUDA_ERROR_INVALID_VALUE;
  DeviceGuard g(hh->device);
  CUCHOL_CHECK(g.err);
  CUCHOL_CHECK(cudaStreamSynchronize(hh->s_copy));
  CUCHOL_CHECK(cudaStreamSynchronize(hh->s_out));
  CUCHOL_CHECK(cudaStreamSynchronize(hh->s_gemm));
  CUCHOL_CHECK(cudaStreamSynchronize(hh->s_tail));
  CUCHOL_CHECK(cudaStreamSynchronize(hh->h->s_panel));
  CUCHOL_CHECK(cudaStreamSynchronize(hh->h->s_update));
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuMultiGPULAPACKGetStats(CUmultiGPULAPACKhandle hh, unsigned long long* launches,
                                                           unsigned long long* h2d_bytes,
                                                           unsigned long long* d2h_bytes) {
  if (hh == nullptr) return CUDA_ERROR_INVALID_VALUE;
  if (launches) *launches = hh->h->launches;
  if (h2d_bytes) *h2d_bytes = hh->h2d_bytes;
  if (d2h_bytes) *d2h_bytes = hh->d2h_bytes;
  return CUDA_SUCCESS;
}

#define CUCHOL_API_HOST(P, T, H)                                                                                  \
  extern "C" CUCHOL_EXPORT CUresult cuMultiGPU##P##potrf(CUmultiGPULAPACKhandle h, CBlasUplo u, size_t n, H* A,  \
                                                         size_t lda, long* info) {                               \
    return host_potrf<T>("cuMultiGPU" #P "potrf", h, u, n, reinterpret_cast<T*>(A), lda, info);                  \
  }                                                                                                               \
  extern "C" CUCHOL_EXPORT CUresult cuMultiGPU##P##trtri(CUmultiGPULAPACKhandle h, CBlasUplo u, CBlasDiag d,     \
                                                         size_t n, H* A, size_t lda, long* info) {               \
    return host_trtri<T>("cuMultiGPU" #P "trtri", h, u, d, n, reinterpret_cast<T*>(A), lda, info);               \
  }                                                                                                               \
  extern "C" CUCHOL_EXPORT CUresult cuMultiGPU##P##lauum(CUmultiGPULAPACKhandle h, CBlasUplo u, size_t n, H* A,  \
                                                         size_t lda, long* info) {                               \
    return host_lauum<T>("cuMultiGPU" #P "lauum", h, u, n, reinterpret_cast<T*>(A), lda, info);                  \
  }                                                                                                               \
  extern "C" CUCHOL_EXPORT CUresult cuMultiGPU##P##potri(CUmultiGPULAPACKhandle h, CBlasUplo u, size_t n, H* A,  \
                                                         size_t lda, long* info) {                               \
    return host_potri<T>("cuMultiGPU" #P "potri", h, u, n, reinterpret_cast<T*>(A), lda, info);                  \
  }
CUCHOL_API_HOST(S, float, float)
CUCHOL_API_HOST(D, double, double)
CUCHOL_API_HOST(C, cuFloatComplex, cucholesky_cfloat)
CUCHOL_API_HOST(Z, cuDoubleComplex, cucholesky_cdouble)
