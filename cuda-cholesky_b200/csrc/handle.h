// Library-internal handle and error plumbing.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/cucholesky_ext.h"

struct __culapackhandle_st {
  int device;
  cudaStream_t s_panel;    // diagonal block, panel solve, lookahead update (high priority)
  cudaStream_t s_update;   // trailing update
  cudaEvent_t ev_panel, ev_update;
  int* d_words;            // device scratch words: [0] info, [1] scan max, [2] scan min,
                           // [3] engine error (a bounded wait gave up)
  int* h_words;            // pinned mirror of d_words
  double* d_logdet;        // [0] fused potrf log det, [1] ?logdet result (double)
  float* d_logdet_f;       // ?logdet result (float)
  double* h_logdet;        // pinned mirror of d_logdet[0]
  double* d_part;          // ?logdet partial sums (kLogdetMaxBlocks)
  unsigned int* d_counter; // ?logdet retirement counter
  void* ws;                // grow-only workspace
  size_t ws_bytes;
  void* desc_dev;          // device copy of grouped-launch problem lists
  void* desc_host;         // pinned staging for them
  size_t desc_bytes, desc_used;
  int num_sms;
  unsigned long long launches;   // kernels launched by this handle
  int force_simt;                // testing: route FP64 products to the SIMT engine
  int wait_limit;                // testing: iterations of the triangular solves' ticket waits
                                 // (< 0: the default limit)
  int potrf_sub;                 // ?potrf outer block in diagonal blocks (0: tuning table)
  int lauum_cols;                // testing: ?lauum block-column width (0: from the workspace cap)
};

namespace cuchol {

constexpr int kLogdetMaxBlocks = 1024;

// CUDA runtime error -> CUresult.  The common codes share their numeric values
// between the runtime and driver enums; the rest are passed through.
inline CUresult to_cu(cudaError_t e) { return static_cast<CUresult>(static_cast<int>(e)); }

const char* error_string(int e);

CUresult report(cudaError_t e, const char* call, const char* func, const char* file, int line);

// Every device allocation of the library (cudaMalloc) goes through here, so that a
// test can make one fail (cuLAPACKFailAllocation) and check that each
// routine reports CUDA_ERROR_OUT_OF_MEMORY and leaves its handle usable.
cudaError_t dev_malloc_bytes(void** p, size_t bytes);
template <typename T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
  return dev_malloc_bytes(reinterpret_cast<void**>(p), bytes);
}

// Grow the handle's workspace to at least `bytes` (synchronises the handle's
// streams first, because queued work may still use the old buffer).
CUresult ensure_workspace(CULAPACKhandle h, size_t bytes);

// Copy `bytes` of problem descriptors into the device list area; returns the
// device address, or nullptr if the area is full.
void* stage_descriptors(CULAPACKhandle h, const void* src, size_t bytes, cudaStream_t s);

}  // namespace cuchol

#define CUCHOL_CHECK(call)                                                              \
  do {                                                                                  \
    cudaError_t e__ = (call);                                                           \
    if (e__ != cudaSuccess) return ::cuchol::report(e__, #call, __func__, __FILE__, __LINE__); \
  } while (0)

#define CUCHOL_CHECK_CU(call)                                                           \
  do {                                                                                  \
    CUresult r__ = (call);                                                              \
    if (r__ != CUDA_SUCCESS) return r__;                                                \
  } while (0)
