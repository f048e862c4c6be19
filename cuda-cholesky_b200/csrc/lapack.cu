// Host drivers of the dense SPD path and the C ABI of include/lapack.h.
//
// All four element types run the same drivers (templates over T).  Upper storage
// is handled by running the lower algorithm on the transposed view of A (element
// (i, j) of the logical lower triangle at A[i*rs + j*cs], (rs, cs) = (lda, 1)), which
// produces U = L^T in place; see diag.cuh.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <type_traits>
#include <vector>

#include "diag.cuh"
#include "dmma.cuh"
#include "gemm.cuh"
#include "zmma.cuh"
#include "handle.h"
#include "panel.cuh"
#include "tc.cuh"
#include "trsm.cuh"
#include "tuning.cuh"

using namespace cuchol;

// ------------------------------------------------------------------------------
// Hooks (reference blas/xerbla.c:5-9, multigpu/error.c:4-11)
// ------------------------------------------------------------------------------
static void default_xerbla(const char* function, long info) {
  fprintf(stderr, "On entry to %s parameter %ld had an invalid value\n", function, info);
}
static void default_error_handler(const char* call, const char* function, const char* file, int line,
                                  int error, const char* (*strerror)(int)) {
  fprintf(stderr, "Error:\n\t%s returned %d (%s) in %s (%s:%d)\n", call, error, strerror(error), function,
          file, line);
}
#define CUCHOL_EXPORT __attribute__((visibility("default")))
extern "C" {
CUCHOL_EXPORT xerbla_t xerbla = &default_xerbla;
CUCHOL_EXPORT errorHandler_t errorHandler = &default_error_handler;
}

namespace cuchol {

const char* error_string(int e) { return cudaGetErrorString(static_cast<cudaError_t>(e)); }

// Allocations still to succeed before one fails (< 0: none fails).
static std::atomic<int> g_fail_after{-1};

cudaError_t dev_malloc_bytes(void** p, size_t bytes) {
  int left = g_fail_after.load();
  while (left >= 0) {
    if (g_fail_after.compare_exchange_weak(left, left - 1)) {
      if (left == 0) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
      }
      break;
    }
  }
  return cudaMalloc(p, bytes);
}

CUresult report(cudaError_t e, const char* call, const char* func, const char* file, int line) {
  if (errorHandler != nullptr) errorHandler(call, func, file, line, (int)e, &error_string);
  return to_cu(e);
}

CUresult ensure_workspace(CULAPACKhandle h, size_t bytes) {
  if (bytes <= h->ws_bytes) return CUDA_SUCCESS;
  CUCHOL_CHECK(cudaStreamSynchronize(h->s_panel));
  CUCHOL_CHECK(cudaStreamSynchronize(h->s_update));
  if (h->ws != nullptr) CUCHOL_CHECK(cudaFree(h->ws));
  h->ws = nullptr;
  h->ws_bytes = 0;
  CUCHOL_CHECK(dev_malloc(&h->ws, bytes));
  h->ws_bytes = bytes;
  return CUDA_SUCCESS;
}

void* stage_descriptors(CULAPACKhandle h, const void* src, size_t bytes, cudaStream_t s) {
  size_t off = (h->desc_used + 255) & ~size_t(255);
  if (off + bytes > h->desc_bytes) return nullptr;
  memcpy(static_cast<char*>(h->desc_host) + off, src, bytes);
  void* dst = static_cast<char*>(h->desc_dev) + off;
  if (cudaMemcpyAsync(dst, static_cast<char*>(h->desc_host) + off, bytes, cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return nullptr;
  h->desc_used = off + bytes;
  return dst;
}

}  // namespace cuchol

namespace {

__global__ void narrow_double_kernel(const double* s, float* d) { *d = (float)*s; }

template <typename T> struct Tune { static constexpr int nb = 128; };   // diagonal block
template <> struct Tune<cuDoubleComplex> { static constexpr int nb = 64; };

template <typename T> constexpr char type_char() {
  return std::is_same<T, float>::value ? 'S' : std::is_same<T, double>::value ? 'D'
       : std::is_same<T, cuFloatComplex>::value ? 'C' : 'Z';
}

inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// ---- tile engine launcher -------------------------------------------------------
template <typename T, int LA, int LB, int TM>
CUresult launch_simt(CULAPACKhandle h, const GemmLaunch<T>& L, int tiles, cudaStream_t s, const int* abort) {
  gemm_simt_kernel<T, LA, LB, TM><<<tiles, 256, 0, s>>>(L, abort);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

template <int LA, int LB>
CUresult launch_dmma_group(CULAPACKhandle h, const GemmLaunch<double>& L, int tiles, cudaStream_t s,
                           const int* abort) {
  gemm_dmma_group_kernel<LA, LB><<<tiles, kDgThreads, 0, s>>>(L, abort);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

template <typename T, int TM = 4>
CUresult launch_dispatch(CULAPACKhandle h, const GemmLaunch<T>& L, int tiles, int la, int lb, cudaStream_t s,
                         const int* abort) {
  if constexpr (std::is_same<T, double>::value && TM == 4) {
    // FP64 on the tensor cores (64 x 64 tiles, numbered as by the SIMT engine)
    if (!h->force_simt) {
      if (la == 0 && lb == 0) return launch_dmma_group<0, 0>(h, L, tiles, s, abort);
      if (la == 0 && lb == 1) return launch_dmma_group<0, 1>(h, L, tiles, s, abort);
      if (la == 1 && lb == 0) return launch_dmma_group<1, 0>(h, L, tiles, s, abort);
      return launch_dmma_group<1, 1>(h, L, tiles, s, abort);
    }
  }
  if (la == 0 && lb == 0) return launch_simt<T, 0, 0, TM>(h, L, tiles, s, abort);
  if (la == 0 && lb == 1) return launch_simt<T, 0, 1, TM>(h, L, tiles, s, abort);
  if (la == 1 && lb == 0) return launch_simt<T, 1, 0, TM>(h, L, tiles, s, abort);
  return launch_simt<T, 1, 1, TM>(h, L, tiles, s, abort);
}

constexpr int kTile = 64;

// ---- FP64 tensor-core path (dmma.cuh) --------------------------------------------
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// FP64 view (rows x k) as a TMA map with 128-byte swizzle; rows / k beyond the
// view read as zero.  Layout R (rows contiguous): 16 x 16 boxes.  Layout K (k
// contiguous): boxes of 16 k x box_rows rows.
bool make_map(CUtensorMap* map, const double* base, int layout, long long rows, long long k, long long ld,
              int box_rows) {
  EncodeTiledFn fn = encode_tiled();
  if (fn == nullptr) return false;
  cuuint64_t dims[2], strides[1] = {(cuuint64_t)ld * sizeof(double)};
  cuuint32_t box[2], estr[2] = {1, 1};
  if (layout == dmma::LAYOUT_R) {
    dims[0] = rows; dims[1] = k; box[0] = 16; box[1] = 16;
  } else {
    dims[0] = k; dims[1] = rows; box[0] = 16; box[1] = box_rows;
  }
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <int LA, int LB, bool TRI, int MB>
CUresult launch_dmma(CULAPACKhandle h, const CUtensorMap& ma, const CUtensorMap& mb, const dmma::Params& q,
                     int tiles, cudaStream_t s, const int* abort) {
  constexpr int smem = dmma::Shape<MB>::SMEM_BYTES;
  static bool attr = false;
  if (!attr) {
    CUCHOL_CHECK(cudaFuncSetAttribute(dmma::gemm_kernel<LA, LB, TRI, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
    // several CTAs per SM: ask for the whole unified L1/shared carve-out
    CUCHOL_CHECK(cudaFuncSetAttribute(dmma::gemm_kernel<LA, LB, TRI, MB>,
                                      cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    attr = true;
  }
  dmma::gemm_kernel<LA, LB, TRI, MB><<<tiles, dmma::THREADS, smem, s>>>(ma, mb, q, abort);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

template <bool TRI, int MB>
CUresult launch_dmma_layouts(CULAPACKhandle h, int la, int lb, const CUtensorMap& ma, const CUtensorMap& mb,
                             const dmma::Params& q, int tiles, cudaStream_t s, const int* abort) {
  if (la == 0 && lb == 0) return launch_dmma<0, 0, TRI, MB>(h, ma, mb, q, tiles, s, abort);
  if (la == 0 && lb == 1) return launch_dmma<0, 1, TRI, MB>(h, ma, mb, q, tiles, s, abort);
  if (la == 1 && lb == 0) return launch_dmma<1, 0, TRI, MB>(h, ma, mb, q, tiles, s, abort);
  return launch_dmma<1, 1, TRI, MB>(h, ma, mb, q, tiles, s, abort);
}

// Warp tile height of the FP64 engine for a problem (m16 blocks per warp): 64 x 64
// tiles, three CTAs per SM, for the updates of the factorizations (k up to about a
// thousand: more resident warps and finer waves measured faster), 128 x 64 tiles,
// two per SM, for long products (fewer operand bytes per flop).
inline int dmma_mb(const GemmProblem<double>& p) { return p.k >= 2048 ? 4 : 2; }

// Runs the problem on the FP64 tensor-core engine if its views fit the engine
// (each view row- or k-contiguous, 16-byte aligned, even leading dimension);
// returns false (nothing launched) otherwise.
bool try_dmma(CULAPACKhandle h, const GemmProblem<double>& p, cudaStream_t s, const int* abort, CUresult* rc) {
  const int la = (p.a_rs == 1) ? dmma::LAYOUT_R : (p.a_ks == 1 ? dmma::LAYOUT_K : -1);
  const int lb = (p.b_rs == 1) ? dmma::LAYOUT_R : (p.b_ks == 1 ? dmma::LAYOUT_K : -1);
  if (la < 0 || lb < 0 || p.k <= 0) return false;
  const long long lda = (la == dmma::LAYOUT_R) ? p.a_ks : p.a_rs;
  const long long ldb = (lb == dmma::LAYOUT_R) ? p.b_ks : p.b_rs;
  if ((lda & 1) || (ldb & 1) || !aligned16(p.a) || !aligned16(p.b)) return false;
  CUtensorMap ma, mb;
  const int mbk = dmma_mb(p), bm = 32 * mbk;
  if (!make_map(&ma, p.a, la, p.m, p.k, lda, bm) || !make_map(&mb, p.b, lb, p.n, p.k, ldb, dmma::BN))
    return false;
  dmma::Params q;
  q.c = p.c; q.c_rs = p.c_rs; q.c_cs = p.c_cs;
  q.cin = p.cin; q.cin_rs = p.cin_rs; q.cin_cs = p.cin_cs;
  q.m = p.m; q.n = p.n; q.k = p.k;
  q.alpha = p.alpha; q.beta = p.beta;
  q.tri_a = p.tri_a; q.tri_b = p.tri_b; q.unit_a = p.unit_a; q.unit_b = p.unit_b;
  q.lower_only = p.lower_only;
  q.tiles_n = (p.n + dmma::BN - 1) / dmma::BN;
  const long long other = (p.c_rs == 1) ? p.c_cs : p.c_rs;
  q.vec_ok = aligned16(p.c) && !(other & 1) &&
             (p.cin == nullptr || (p.cin == p.c && p.cin_rs == p.c_rs && p.cin_cs == p.c_cs));
  q.preload = (p.alpha == 1.0 || p.alpha == -1.0) &&
              (p.cin == nullptr || (p.cin_rs == p.c_rs && p.cin_cs == p.c_cs) || p.cin != p.c);
  q.neg = q.preload && p.alpha == -1.0;
  q.err = h->d_words + 3;
  q.tiles_m = (p.m + bm - 1) / bm;
  const int all_tiles = q.tiles_m * q.tiles_n;
  // one tile per CTA: several tiles per CTA measured slower (tails, uneven skipping)
  const int tiles = all_tiles;
  const bool tri = p.tri_a || p.tri_b || p.unit_a || p.unit_b;
  if (mbk == 2)
    *rc = tri ? launch_dmma_layouts<true, 2>(h, la, lb, ma, mb, q, tiles, s, abort)
              : launch_dmma_layouts<false, 2>(h, la, lb, ma, mb, q, tiles, s, abort);
  else
    *rc = tri ? launch_dmma_layouts<true, 4>(h, la, lb, ma, mb, q, tiles, s, abort)
              : launch_dmma_layouts<false, 4>(h, la, lb, ma, mb, q, tiles, s, abort);
  return true;
}

// ---- complex FP64 tensor-core path (zmma.cuh) -------------------------------------
// A complex view as an FP64 TMA map (128-byte swizzle): layout R (rows contiguous)
// is the real matrix of 2 * rows x k doubles, boxes of 16 doubles (8 complex rows)
// x 8 k; layout K (k contiguous) is rows x 2k doubles, boxes of 16 doubles (8
// complex k) x box_rows rows.  Any leading dimension works: its byte stride is a
// multiple of 16.
bool make_zmap(CUtensorMap* map, const cuDoubleComplex* base, int layout, long long rows, long long k,
               long long ld, int box_rows) {
  EncodeTiledFn fn = encode_tiled();
  if (fn == nullptr) return false;
  cuuint64_t dims[2], strides[1] = {(cuuint64_t)ld * sizeof(cuDoubleComplex)};
  cuuint32_t box[2], estr[2] = {1, 1};
  if (layout == dmma::LAYOUT_R) {
    dims[0] = 2 * rows; dims[1] = k; box[0] = 16; box[1] = zmma::BK;
  } else {
    dims[0] = 2 * k; dims[1] = rows; box[0] = 16; box[1] = box_rows;
  }
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<cuDoubleComplex*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int LA, int LB, bool TRI, int MB>
CUresult launch_zmma(CULAPACKhandle h, const CUtensorMap& ma, const CUtensorMap& mb, const zmma::Params& q,
                     int tiles, cudaStream_t s, const int* abort) {
  constexpr int smem = zmma::Shape<MB>::SMEM_BYTES;
  static bool attr = false;
  if (!attr) {
    CUCHOL_CHECK(cudaFuncSetAttribute(zmma::gemm_kernel<LA, LB, TRI, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
    CUCHOL_CHECK(cudaFuncSetAttribute(zmma::gemm_kernel<LA, LB, TRI, MB>,
                                      cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    attr = true;
  }
  zmma::gemm_kernel<LA, LB, TRI, MB><<<tiles, zmma::THREADS, smem, s>>>(ma, mb, q, abort);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

template <bool TRI, int MB>
CUresult launch_zmma_layouts(CULAPACKhandle h, int la, int lb, const CUtensorMap& ma, const CUtensorMap& mb,
                             const zmma::Params& q, int tiles, cudaStream_t s, const int* abort) {
  if (la == 0 && lb == 0) return launch_zmma<0, 0, TRI, MB>(h, ma, mb, q, tiles, s, abort);
  if (la == 0 && lb == 1) return launch_zmma<0, 1, TRI, MB>(h, ma, mb, q, tiles, s, abort);
  if (la == 1 && lb == 0) return launch_zmma<1, 0, TRI, MB>(h, ma, mb, q, tiles, s, abort);
  return launch_zmma<1, 1, TRI, MB>(h, ma, mb, q, tiles, s, abort);
}

// Warp tile height of the complex engine for a problem (m16 blocks per warp): 32 x 64
// tiles, three CTAs per SM, for k < 1024 (the updates of zpotrf up to n = 16384: their
// CTAs retire twice as often, so the panel chain finds SMs sooner; zpotrf n = 8192
// 38.2 -> 36.9 ms, n = 4096 9.7 -> 8.7 ms), 64 x 64 otherwise.
constexpr int kZmmaShortK = 1024;
inline int zmma_mb(const GemmProblem<cuDoubleComplex>& p) { return p.k < kZmmaShortK ? 1 : 2; }

// Runs a complex double problem on the FP64 tensor-core engine when both operand
// views are row- or k-contiguous and 16-byte aligned; false (nothing launched)
// otherwise.
bool try_zmma(CULAPACKhandle h, const GemmProblem<cuDoubleComplex>& p, cudaStream_t s, const int* abort,
              CUresult* rc) {
  const int la = (p.a_rs == 1) ? dmma::LAYOUT_R : (p.a_ks == 1 ? dmma::LAYOUT_K : -1);
  const int lb = (p.b_rs == 1) ? dmma::LAYOUT_R : (p.b_ks == 1 ? dmma::LAYOUT_K : -1);
  if (la < 0 || lb < 0 || p.k <= 0) return false;
  const long long lda = (la == dmma::LAYOUT_R) ? p.a_ks : p.a_rs;
  const long long ldb = (lb == dmma::LAYOUT_R) ? p.b_ks : p.b_rs;
  if (!aligned16(p.a) || !aligned16(p.b)) return false;
  CUtensorMap ma, mb;
  const int mbk = zmma_mb(p), bm = 32 * mbk;
  if (!make_zmap(&ma, p.a, la, p.m, p.k, lda, bm) || !make_zmap(&mb, p.b, lb, p.n, p.k, ldb, zmma::BN))
    return false;
  zmma::Params q;
  q.c = p.c; q.c_rs = p.c_rs; q.c_cs = p.c_cs;
  q.cin = p.cin; q.cin_rs = p.cin_rs; q.cin_cs = p.cin_cs;
  q.m = p.m; q.n = p.n; q.k = p.k;
  q.alpha = p.alpha; q.beta = p.beta;
  q.conj_a = p.conj_a; q.conj_b = p.conj_b;
  q.tri_a = p.tri_a; q.tri_b = p.tri_b; q.unit_a = p.unit_a; q.unit_b = p.unit_b;
  q.lower_only = p.lower_only; q.real_diag = p.real_diag;
  q.tiles_m = (p.m + bm - 1) / bm;
  q.tiles_n = (p.n + zmma::BN - 1) / zmma::BN;
  const bool unit_alpha = p.alpha.y == 0.0 && (p.alpha.x == 1.0 || p.alpha.x == -1.0);
  q.preload = unit_alpha &&
              (p.cin == nullptr || (p.cin_rs == p.c_rs && p.cin_cs == p.c_cs) || p.cin != p.c);
  q.neg = q.preload && p.alpha.x == -1.0;
  q.err = h->d_words + 3;
  const int tiles = q.tiles_m * q.tiles_n;
  const bool tri = p.tri_a || p.tri_b || p.unit_a || p.unit_b;
  if (mbk == 1)
    *rc = tri ? launch_zmma_layouts<true, 1>(h, la, lb, ma, mb, q, tiles, s, abort)
              : launch_zmma_layouts<false, 1>(h, la, lb, ma, mb, q, tiles, s, abort);
  else
    *rc = tri ? launch_zmma_layouts<true, 2>(h, la, lb, ma, mb, q, tiles, s, abort)
              : launch_zmma_layouts<false, 2>(h, la, lb, ma, mb, q, tiles, s, abort);
  return true;
}

template <typename T>
CUresult gemm(CULAPACKhandle h, GemmProblem<T> p, cudaStream_t s, const int* abort) {
  if (p.m <= 0 || p.n <= 0) return CUDA_SUCCESS;
  if constexpr (std::is_same<T, double>::value) {
    CUresult rc;
    if (!h->force_simt && try_dmma(h, p, s, abort, &rc)) return rc;
  }
  if constexpr (std::is_same<T, cuDoubleComplex>::value) {
    CUresult rc;
    if (!h->force_simt && try_zmma(h, p, s, abort, &rc)) return rc;
  }
  GemmLaunch<T> L{};
  L.list = nullptr;
  L.nlist = 0;
  p.tile_begin = 0;
  if constexpr (std::is_same<T, float>::value) {
    // large FP32 products: 128 x 128 tiles, except the factorization's lower-only
    // updates with k = 256, which stay on 64 x 64 tiles (more CTAs per SM to hide their
    // short k loop).  Measured at n = 16384: spotri 335 -> 179 ms, spotrf unchanged.
    if (p.m >= 256 && p.n >= 256 && (p.k >= 512 || (!p.lower_only && p.k >= 64))) {
      constexpr int big = 128;
      p.tiles_n = (p.n + big - 1) / big;
      L.single = p;
      return launch_dispatch<T, 8>(h, L, ((p.m + big - 1) / big) * p.tiles_n, p.a_rs == 1 ? 0 : 1,
                                   p.b_rs == 1 ? 0 : 1, s, abort);
    }
  }
  p.tiles_n = (p.n + kTile - 1) / kTile;
  const int tiles = ((p.m + kTile - 1) / kTile) * p.tiles_n;
  L.single = p;
  return launch_dispatch<T>(h, L, tiles, p.a_rs == 1 ? 0 : 1, p.b_rs == 1 ? 0 : 1, s, abort);
}

// All problems must share the contiguity of their views.
template <typename T>
CUresult gemm_group(CULAPACKhandle h, std::vector<GemmProblem<T>>& ps, cudaStream_t s, const int* abort) {
  if (ps.empty()) return CUDA_SUCCESS;
  int tiles = 0;
  for (auto& p : ps) {
    p.tiles_n = (p.n + kTile - 1) / kTile;
    p.tile_begin = tiles;
    tiles += ((p.m + kTile - 1) / kTile) * p.tiles_n;
  }
  // few problems: one launch each, so FP64 ones reach the tensor-core engine
  if (ps.size() <= 8) {
    for (auto& p : ps) CUCHOL_CHECK_CU(gemm<T>(h, p, s, abort));
    return CUDA_SUCCESS;
  }
  void* dev = stage_descriptors(h, ps.data(), ps.size() * sizeof(GemmProblem<T>), s);
  if (dev == nullptr) {   // list area full: one launch per problem
    for (auto& p : ps) CUCHOL_CHECK_CU(gemm<T>(h, p, s, abort));
    return CUDA_SUCCESS;
  }
  GemmLaunch<T> L{};
  L.list = static_cast<const GemmProblem<T>*>(dev);
  L.nlist = (int)ps.size();
  return launch_dispatch<T>(h, L, tiles, ps[0].a_rs == 1 ? 0 : 1, ps[0].b_rs == 1 ? 0 : 1, s, abort);
}

template <typename T>
GemmProblem<T> problem() {
  GemmProblem<T> p;
  memset(&p, 0, sizeof(p));
  p.alpha = from_real<T>(RealOf<T>(1));
  p.beta = zero<T>();
  return p;
}

template <typename T>
CUresult copy_view(CULAPACKhandle h, const T* src, long long s_rs, long long s_cs, T* dst, long long d_rs, long long d_cs, int m,
                   int n, bool lower_only, cudaStream_t s, const int* abort) {
  if (m <= 0 || n <= 0) return CUDA_SUCCESS;
  dim3 grid((m + 31) / 32, (n + 31) / 32);
  copy_view_kernel<T><<<grid, 256, 0, s>>>(src, s_rs, s_cs, dst, d_rs, d_cs, m, n, lower_only ? 1 : 0, abort);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

// A bounded wait inside an engine kernel gave up (h_words mirrors d_words):
// report it as a launch timeout and clear the word for the next call.
CUresult check_engine(CULAPACKhandle h) {
  if (h->h_words[3] == 0) return CUDA_SUCCESS;
  h->h_words[3] = 0;
  CUCHOL_CHECK(cudaMemset(h->d_words + 3, 0, sizeof(int)));
  if (errorHandler != nullptr)
    errorHandler("engine wait", __func__, __FILE__, __LINE__, (int)CUDA_ERROR_LAUNCH_TIMEOUT, &error_string);
  return CUDA_ERROR_LAUNCH_TIMEOUT;
}

template <typename T>
CUresult set_smem(const void* fn, size_t bytes) {
  CUCHOL_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return CUDA_SUCCESS;
}

// ---- FP32 updates on the TF32 tensor cores, split in three (tc.cuh, SPLIT3) -------
// C -= Q(r) Q(c)^T on the logical lower trapezoid m x ncols whose corner is the
// diagonal element (r0, r0) of A (column-major, lda), with Q = qhi + qlo k-major (row
// pitch ldq, q_rows rows): operand rows from qrow, k columns [koff, koff + k).  Upper
// storage (rs = lda) writes the same symmetric update into the physical upper
// trapezoid.  The caller checks the alignment rules (tc3_usable).
bool tc3_usable(const float* A, long long lda) { return aligned16(A) && (lda % 4) == 0; }

CUresult tc3_update(CULAPACKhandle h, const float* qhi, const float* qlo, long long ldq, int q_rows, int qrow,
                    int koff, int k, float* A, long long lda, bool upper, int r0, int m, int ncols, cudaStream_t s,
                    const int* stop) {
  if (m <= 0 || ncols <= 0 || k <= 0) return CUDA_SUCCESS;
  EncodeTiledFn fn = encode_tiled();
  if (fn == nullptr) return CUDA_ERROR_NOT_SUPPORTED;
  CUtensorMap mhi, mlo, mc;
  const cuuint32_t es[2] = {1, 1};
  const cuuint64_t qdims[2] = {(cuuint64_t)k, (cuuint64_t)q_rows};
  const cuuint64_t qstr[1] = {(cuuint64_t)ldq * sizeof(float)};
  const cuuint32_t qbox[2] = {(cuuint32_t)tc::OpKind<float>::BK, (cuuint32_t)tc::BM};
  for (int w = 0; w < 2; ++w) {
    const float* q = (w == 0 ? qhi : qlo) + koff;
    if (fn(w == 0 ? &mhi : &mlo, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(q), qdims, qstr, qbox, es,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return CUDA_ERROR_INVALID_VALUE;
  }
  float* corner = A + (long long)r0 * (lda + 1);
  const cuuint64_t cdims[2] = {(cuuint64_t)(upper ? ncols : m), (cuuint64_t)(upper ? m : ncols)};
  const cuuint64_t cstr[1] = {(cuuint64_t)lda * sizeof(float)};
  const cuuint32_t cbox[2] = {32, 32};
  if (fn(&mc, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, corner, cdims, cstr, cbox, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
         upper ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return CUDA_ERROR_INVALID_VALUE;
  tc::Params prm{};
  prm.m = m;
  prm.n = ncols;
  prm.k = k;
  prm.a_row0 = qrow;
  prm.b_row0 = qrow;
  prm.alpha = -1.f;
  prm.lower_only = 1;
  prm.tiles_m = (m + tc::BM - 1) / tc::BM;
  prm.tiles_n = (ncols + tc::BN - 1) / tc::BN;
  prm.err = h->d_words + 3;
  const int tiles = prm.tiles_n * (prm.tiles_n + 1) / 2 + (prm.tiles_m - prm.tiles_n) * prm.tiles_n;
  constexpr int smem = tc::Ring<true>::SMEM;
  static bool attr[2] = {false, false};
  if (!attr[upper]) {
    CUCHOL_CHECK(cudaFuncSetAttribute(upper ? (const void*)tc::update_kernel<float, true, true>
                                            : (const void*)tc::update_kernel<float, true, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr[upper] = true;
  }
  if (upper)
    tc::update_kernel<float, true, true><<<tiles, tc::THREADS, smem, s>>>(mhi, mlo, mc, prm, stop);
  else
    tc::update_kernel<float, true, false><<<tiles, tc::THREADS, smem, s>>>(mhi, mlo, mc, prm, stop);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

// ---- ?POTRF ---------------------------------------------------------------------
// Right-looking blocked Cholesky, outer blocks of NB = sub*nb columns (each factored
// as sub nb-wide sub-panels; sub from the tuning table, 2 to 8 by n for FP64),
// lookahead depth 1, on two streams:
//   panel stream : for each sub-panel: diagonal-block factor -> row-parallel panel
//                  solve (into A and the packed buffer P) -> the update of the outer
//                  block's remaining sub-panel columns by it.  Then [wait previous
//                  trailing update] -> update of the next outer block (lookahead,
//                  k = NB)
//   update stream: [wait panel] -> update of the rest of the trailing matrix (k = NB)
// The next outer block is factored on a few SMs while the trailing update of the
// previous one runs on the rest; a wider outer block cuts the trailing update's
// tiles per flop (their fill and drain are the engine's overhead) at the price of
// more panel-stream work per step, so the best width grows with n.
// P (ping-pong pair) holds rows from the first sub-panel's diagonal block down:
// P(r, c) = L(j + nb + r, j + c).  Failure: the diagonal kernel sets the device
// info word, and every later kernel exits at entry when it is set.
constexpr int kDiagThreads2 = 256;

// `on_final`, when given, is called once per diagonal block c .. c + jb - 1 in
// order, as soon as the queued work that finishes that block column of the factor
// (logical rows c .. n-1) has been issued, with the stream that work is on: a
// caller can queue the copy of those columns behind it (host-memory routines).
// `ncols` < n factors only the leading ncols columns of the n x n trailing matrix
// (a tall panel: its diagonal blocks, the solves below them, and the updates of its
// own columns); the columns right of it are neither read nor written.
using FinalColumns = std::function<CUresult(int c, int jb, cudaStream_t s)>;

template <typename T>
CUresult potrf_run(CULAPACKhandle h, bool upper, int n, T* A, long long lda, long* info, double* logdet_out,
                   const FinalColumns* on_final = nullptr, int ncols = -1) {
  if (ncols < 0 || ncols > n) ncols = n;
  constexpr int nb = Tune<T>::nb;
  // outer block: sub diagonal blocks, from the handle's override or the tuning table
  const int NB = (h->potrf_sub > 0 ? h->potrf_sub : tuned_potrf_sub(type_char<T>(), n)) * nb;
  using Smem = DiagSmem<T, nb>;
  const long long rs = upper ? lda : 1, cs = upper ? 1 : lda;
  auto at = [&](long long i, long long j) { return A + i * rs + j * cs; };
  cudaStream_t sp = h->s_panel, su = h->s_update;
  int* d_info = h->d_words;

  const long long ldp = (long long)round_up((size_t)n, 2);
  // FP32 with an aligned A: the updates run on the TF32 tensor cores as split
  // products, from hi / lo copies of the solved panel in k-major buffers Q (row
  // r = P row r, pitch ldq), ping-pong like P; P itself is then not needed
  bool tc3 = false;
  if constexpr (std::is_same<T, float>::value) tc3 = !h->force_simt && tc3_usable(A, lda) && n > 128;
  const long long ldq = (long long)round_up((size_t)NB, 32);
  const size_t ws = tc3 ? sizeof(T) * 4 * (size_t)n * ldq : sizeof(T) * (2 * (size_t)ldp * NB);
  CUCHOL_CHECK_CU(ensure_workspace(h, ws));
  T* pbuf[2] = {static_cast<T*>(h->ws), static_cast<T*>(h->ws) + (size_t)ldp * NB};
  T* qbuf[4] = {static_cast<T*>(h->ws), static_cast<T*>(h->ws) + (size_t)n * ldq,
                static_cast<T*>(h->ws) + 2 * (size_t)n * ldq, static_cast<T*>(h->ws) + 3 * (size_t)n * ldq};

  CUCHOL_CHECK_CU(set_smem<T>((const void*)diag_factor_kernel<T, nb, kDiagThreads2>, Smem::bytes));
  // the panel solve is a row-parallel triangular solve (no inverse of the diagonal
  // block) that writes the solved rows into A and into P
  CUCHOL_CHECK_CU(set_smem<T>((const void*)trsm_rows_kernel<T, T, T, T, OUT_CONVERT>, trsm_rows_smem<T>()));
  if constexpr (std::is_same<T, float>::value)
    CUCHOL_CHECK_CU(set_smem<T>((const void*)trsm_rows_kernel<T, T, T, T, OUT_SPLIT>, trsm_rows_smem<T>()));
  CUCHOL_CHECK(cudaMemsetAsync(d_info, 0, sizeof(int), sp));
  CUCHOL_CHECK(cudaMemsetAsync(h->d_logdet, 0, sizeof(double), sp));
  // the update stream starts after the panel stream's initialisation
  CUCHOL_CHECK(cudaEventRecord(h->ev_panel, sp));
  CUCHOL_CHECK(cudaStreamWaitEvent(su, h->ev_panel, 0));
  CUCHOL_CHECK(cudaEventRecord(h->ev_update, su));

  const T minus_one = from_real<T>(RealOf<T>(-1)), one = from_real<T>(RealOf<T>(1));
  // C -= Phat Phat^H on the lower trapezoid m x ncols of A with its corner on the
  // diagonal at r0; operand rows from P row prow (both sides), k columns [koff, koff + k)
  auto update = [&](const T* P, const T* Qh, const T* Ql, int r0, int m, int ncols, int prow, int koff, int k,
                    cudaStream_t s) -> CUresult {
    if constexpr (std::is_same<T, float>::value) {
      if (tc3)
        return tc3_update(h, Qh, Ql, ldq, n, prow, koff, k, A, lda, upper, r0, m, ncols, s, d_info);
    }
    const T* pa = P + prow + (long long)koff * ldp;
    GemmProblem<T> u = problem<T>();
    u.a = pa; u.a_rs = 1; u.a_ks = ldp;
    u.b = pa; u.b_rs = 1; u.b_ks = ldp; u.conj_b = 1;
    u.c = at(r0, r0); u.c_rs = rs; u.c_cs = cs;
    u.cin = u.c; u.cin_rs = rs; u.cin_cs = cs;
    u.alpha = minus_one; u.beta = one;
    u.lower_only = 1; u.real_diag = 1;
    u.m = m; u.n = ncols; u.k = k;
    return gemm<T>(h, u, s, d_info);
  };

  for (int j = 0, step = 0; j < ncols; j += NB, ++step) {
    const int jB = std::min(NB, ncols - j);
    const int m = n - j - jB;                    // rows below the outer block
    const int mc = ncols - j - jB;               // columns right of it (in the panel)
    T* P = pbuf[step & 1];
    T* Qh = qbuf[2 * (step & 1)];
    T* Ql = qbuf[2 * (step & 1) + 1];
    for (int s0 = 0; s0 < jB; s0 += nb) {
      const int c = j + s0, jb = std::min(nb, j + jB - c);
      const int mr = n - c - jb;                 // rows below this diagonal block
      diag_factor_kernel<T, nb, kDiagThreads2><<<1, kDiagThreads2, Smem::bytes, sp>>>(
          at(c, c), rs, cs, jb, nullptr, nb, c, d_info, h->d_logdet);
      ++h->launches;
      CUCHOL_CHECK(cudaGetLastError());
      if (mr == 0) {
        if (on_final) CUCHOL_CHECK_CU((*on_final)(c, jb, sp));
        break;
      }
      // panel solve into P: rows c + jb .. n-1 are P rows s0 .. (P starts at j + nb)
      // row-parallel triangular solve: A21 := A21 L11^-H in place, and into P (or its
      // hi / lo split into Q)
      bool split = false;
      if constexpr (std::is_same<T, float>::value) {
        if (tc3) {
          const long long qo = (long long)s0 * ldq + s0;
          trsm_rows_kernel<T, T, T, T, OUT_SPLIT><<<(mr + 63) / 64, 256, trsm_rows_smem<T>(), sp>>>(
              at(c + jb, c), rs, cs, mr, jb, at(c, c), rs, cs, Qh + qo, ldq, 1, d_info, Ql + qo);
          split = true;
        }
      }
      if (!split) {
        T* Ps = P + s0 + (long long)s0 * ldp;
        trsm_rows_kernel<T, T, T, T, OUT_CONVERT><<<(mr + 63) / 64, 256, trsm_rows_smem<T>(), sp>>>(
            at(c + jb, c), rs, cs, mr, jb, at(c, c), rs, cs, Ps, 1, ldp, d_info, nullptr);
      }
      ++h->launches;
      CUCHOL_CHECK(cudaGetLastError());
      CUCHOL_CHECK(cudaEventRecord(h->ev_panel, sp));
      if (on_final) CUCHOL_CHECK_CU((*on_final)(c, jb, sp));
      if (s0 + nb < jB) {
        // the outer block's remaining sub-panel columns (rows c + nb .., P rows s0 ..)
        // by this one (k columns s0 .. s0 + nb)
        CUCHOL_CHECK_CU(update(P, Qh, Ql, c + nb, n - c - nb, jB - s0 - nb, s0, s0, nb, sp));
      }
    }
    if (m == 0 || mc == 0) break;
    // lookahead: next outer block (P rows from j + NB, k = jB), after the previous
    // trailing update
    const int jB2 = std::min(NB, mc);
    const int pt = NB - nb;              // P row of global row j + NB
    CUCHOL_CHECK(cudaStreamWaitEvent(sp, h->ev_update, 0));
    CUCHOL_CHECK_CU(update(P, Qh, Ql, j + NB, m, jB2, pt, 0, jB, sp));
    // rest of the trailing matrix, once P holds both sub-panels
    CUCHOL_CHECK(cudaStreamWaitEvent(su, h->ev_panel, 0));
    if (mc > jB2)
      CUCHOL_CHECK_CU(update(P, Qh, Ql, j + NB + jB2, m - jB2, mc - jB2, pt + jB2, 0, jB, su));
    // always recorded: it also covers the copies that still read P
    CUCHOL_CHECK(cudaEventRecord(h->ev_update, su));
  }
  CUCHOL_CHECK(cudaEventRecord(h->ev_update, su));
  CUCHOL_CHECK(cudaStreamWaitEvent(sp, h->ev_update, 0));
  CUCHOL_CHECK(cudaMemcpyAsync(h->h_words, d_info, 4 * sizeof(int), cudaMemcpyDeviceToHost, sp));
  CUCHOL_CHECK(cudaMemcpyAsync(h->h_logdet, h->d_logdet, sizeof(double), cudaMemcpyDeviceToHost, sp));
  CUCHOL_CHECK(cudaStreamSynchronize(sp));
  CUCHOL_CHECK_CU(check_engine(h));
  *info = h->h_words[0];
  if (logdet_out != nullptr) *logdet_out = h->h_logdet[0];
  return CUDA_SUCCESS;
}

// ---- ?TRTRI ---------------------------------------------------------------------
// Recursive in-place inverse of the logical lower triangle:
//   [T11 0; T21 T22]^-1 = [T11^-1 0; -T22^-1 T21 T11^-1, T22^-1]
// All nb x nb diagonal blocks are inverted in one launch, then the tree of splits
// is walked bottom-up; every node of the same height is one grouped launch of
//   X = T22^-1 T21       (TRMM, into workspace)
//   T21 = -X T11^-1      (TRMM, back into A)
// The first zero pivot is located before anything is modified: for lower storage
// the reference's scan runs from the last column back (lapack/dtrtri.c:70-76), so
// info is the largest zero position; for upper it is the smallest.
struct Node { int o, s, s1, height; };

int build_tree(int o, int s, int nb, std::vector<Node>& out) {
  if (s <= nb) return 0;
  int s1 = ((s / nb + 1) / 2) * nb;
  int h1 = build_tree(o, s1, nb, out);
  int h2 = build_tree(o + s1, s - s1, nb, out);
  int hgt = 1 + std::max(h1, h2);
  out.push_back({o, s, s1, hgt});
  return hgt;
}

template <typename T>
CUresult trtri_run(CULAPACKhandle h, bool upper, bool unit, int n, T* A, long long lda, long* info) {
  const int nb = Tune<T>::nb;
  const long long rs = upper ? lda : 1, cs = upper ? 1 : lda;
  auto at = [&](long long i, long long j) { return A + i * rs + j * cs; };
  cudaStream_t sp = h->s_panel;
  *info = 0;
  if (!unit) {
    int init[3] = {0, 0, INT_MAX};
    CUCHOL_CHECK(cudaMemcpyAsync(h->d_words, init, sizeof(init), cudaMemcpyHostToDevice, sp));
    diag_scan_kernel<T><<<std::min((n + 255) / 256, 1024), 256, 0, sp>>>(A, rs + cs, n, h->d_words + 1);
    ++h->launches;
    CUCHOL_CHECK(cudaGetLastError());
    CUCHOL_CHECK(cudaMemcpyAsync(h->h_words, h->d_words, 3 * sizeof(int), cudaMemcpyDeviceToHost, sp));
    CUCHOL_CHECK(cudaStreamSynchronize(sp));
    if (h->h_words[1] != 0) {
      *info = upper ? h->h_words[2] : h->h_words[1];
      return CUDA_SUCCESS;
    }
  }
  constexpr int NB = Tune<T>::nb;
  CUCHOL_CHECK_CU(set_smem<T>((const void*)diag_invert_kernel<T, NB, kDiagThreads2>, DiagSmem<T, NB>::bytes));
  diag_invert_kernel<T, NB, kDiagThreads2><<<(n + nb - 1) / nb, kDiagThreads2, DiagSmem<T, NB>::bytes, sp>>>(
      A, rs, cs, n, nb, unit ? 1 : 0);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());

  std::vector<Node> nodes;
  const int height = build_tree(0, n, nb, nodes);
  // workspace: X blocks of all nodes of one height side by side
  size_t need = 0;
  for (int hh = 1; hh <= height; ++hh) {
    size_t lvl = 0;
    for (auto& nd : nodes)
      if (nd.height == hh) lvl += round_up((size_t)(nd.s - nd.s1), 2) * nd.s1;
    need = std::max(need, lvl);
  }
  CUCHOL_CHECK_CU(ensure_workspace(h, sizeof(T) * std::max<size_t>(need, 1)));
  h->desc_used = 0;
  T* X = static_cast<T*>(h->ws);
  for (int hh = 1; hh <= height; ++hh) {
    std::vector<GemmProblem<T>> p1, p2;
    size_t off = 0;
    for (auto& nd : nodes) {
      if (nd.height != hh) continue;
      const int s1 = nd.s1, s2 = nd.s - nd.s1, o = nd.o;
      const long long ldx = (long long)round_up((size_t)s2, 2);
      T* x = X + off;
      off += (size_t)ldx * s1;
      GemmProblem<T> a = problem<T>();   // X = T22^-1 * T21
      a.a = at(o + s1, o + s1); a.a_rs = rs; a.a_ks = cs; a.tri_a = TRI_LOWER; a.unit_a = unit;
      a.b = at(o + s1, o); a.b_rs = cs; a.b_ks = rs;
      a.c = x; a.c_rs = 1; a.c_cs = ldx;
      a.m = s2; a.n = s1; a.k = s2;
      p1.push_back(a);
      GemmProblem<T> b = problem<T>();   // T21 = -X * T11^-1
      b.a = x; b.a_rs = 1; b.a_ks = ldx;
      b.b = at(o, o); b.b_rs = cs; b.b_ks = rs; b.tri_b = TRI_UPPER; b.unit_b = unit;
      b.c = at(o + s1, o); b.c_rs = rs; b.c_cs = cs;
      b.alpha = from_real<T>(RealOf<T>(-1));
      b.m = s2; b.n = s1; b.k = s1;
      p2.push_back(b);
    }
    CUCHOL_CHECK_CU(gemm_group<T>(h, p1, sp, nullptr));
    CUCHOL_CHECK_CU(gemm_group<T>(h, p2, sp, nullptr));
  }
  CUCHOL_CHECK(cudaStreamSynchronize(sp));
  return CUDA_SUCCESS;
}

// ---- ?LAUUM ---------------------------------------------------------------------
// L^H L (lower; U U^H upper via the transposed view), in place.  The lower part of
// the result, C(i, j) = sum_{k >= i} conj(L(k, i)) L(k, j) for i >= j, reads only
// columns >= j of L.  So the block columns of C are formed left to right, each as one
// product into workspace and then copied over the same block column of A: the
// columns a later block reads are still untouched when it runs.  The block width w
// keeps the workspace ((n - j0) x w) within kLauumWorkspace bytes; orders whose
// whole product fits take one launch.
constexpr size_t kLauumWorkspace = size_t(512) << 20;

template <typename T>
int lauum_width(CULAPACKhandle h, int n) {
  if (h->lauum_cols > 0) return std::min(h->lauum_cols, n);
  const size_t cols = kLauumWorkspace / (sizeof(T) * round_up((size_t)n, 2));
  if (cols >= (size_t)n) return n;
  return (int)std::max<size_t>(256, cols / 256 * 256);
}

template <typename T>
CUresult lauum_run(CULAPACKhandle h, bool upper, int n, T* A, long long lda) {
  const long long rs = upper ? lda : 1, cs = upper ? 1 : lda;
  auto at = [&](long long i, long long j) { return A + i * rs + j * cs; };
  cudaStream_t sp = h->s_panel;
  const int w = lauum_width<T>(h, n);
  const long long ldw = (long long)round_up((size_t)n, 2);
  CUCHOL_CHECK_CU(ensure_workspace(h, sizeof(T) * (size_t)ldw * w));
  T* W = static_cast<T*>(h->ws);
  for (int j0 = 0; j0 < n; j0 += w) {
    const int cols = std::min(w, n - j0), m = n - j0;
    // C(i', j') = sum_k' conj(L(j0 + k', j0 + i')) L(j0 + k', j0 + j'),  k' >= i' >= j'
    GemmProblem<T> p = problem<T>();
    p.a = at(j0, j0); p.a_rs = cs; p.a_ks = rs; p.conj_a = 1; p.tri_a = TRI_UPPER;
    p.b = at(j0, j0); p.b_rs = cs; p.b_ks = rs; p.tri_b = TRI_UPPER;
    p.c = W; p.c_rs = 1; p.c_cs = ldw;
    p.m = m; p.n = cols; p.k = m;
    p.lower_only = 1; p.real_diag = 1;
    CUCHOL_CHECK_CU(gemm<T>(h, p, sp, nullptr));
    CUCHOL_CHECK_CU(copy_view<T>(h, W, 1, ldw, at(j0, j0), rs, cs, m, cols, true, sp, nullptr));
  }
  CUCHOL_CHECK(cudaStreamSynchronize(sp));
  return CUDA_SUCCESS;
}

// ---- ?TRTI22 (single block, caller stream, device info word) ---------------------
template <typename T>
CUresult trti22_run(CULAPACKhandle h, bool upper, bool unit, int n, const T* A, long long lda, T* B,
                    long long ldb, int* dinfo, cudaStream_t stream) {
  const long long ars = upper ? lda : 1, acs = upper ? 1 : lda;
  const long long brs = upper ? ldb : 1, bcs = upper ? 1 : ldb;
  const int nb = Tune<T>::nb;
  if (n > nb) return CUDA_ERROR_INVALID_VALUE;
  // info: zero pivots in the reference's scan order, then (if none) invert
  int init[3] = {0, 0, INT_MAX};
  CUCHOL_CHECK(cudaMemcpyAsync(h->d_words, init, sizeof(init), cudaMemcpyHostToDevice, stream));
  if (!unit) {
    diag_scan_kernel<T><<<1, 128, 0, stream>>>(A, ars + acs, n, h->d_words + 1);
    ++h->launches;
    CUCHOL_CHECK(cudaGetLastError());
  }
  CUCHOL_CHECK(cudaMemcpyAsync(h->h_words, h->d_words, 3 * sizeof(int), cudaMemcpyDeviceToHost, stream));
  CUCHOL_CHECK(cudaStreamSynchronize(stream));
  int inf = (h->h_words[1] == 0) ? 0 : (upper ? h->h_words[2] : h->h_words[1]);
  CUCHOL_CHECK(cudaMemcpyAsync(dinfo, &inf, sizeof(int), cudaMemcpyHostToDevice, stream));
  CUCHOL_CHECK(cudaStreamSynchronize(stream));
  if (inf != 0) return CUDA_SUCCESS;
  if (A != B) CUCHOL_CHECK_CU(copy_view<T>(h, A, ars, acs, B, brs, bcs, n, n, true, stream, nullptr));
  constexpr int NB = Tune<T>::nb;
  CUCHOL_CHECK_CU(set_smem<T>((const void*)diag_invert_kernel<T, NB, kDiagThreads2>, DiagSmem<T, NB>::bytes));
  diag_invert_kernel<T, NB, kDiagThreads2><<<1, kDiagThreads2, DiagSmem<T, NB>::bytes, stream>>>(
      B, brs, bcs, n, n, unit ? 1 : 0);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

// ---- ?LOGDET --------------------------------------------------------------------
template <typename T, typename Out>
CUresult logdet_run(CULAPACKhandle h, const T* x, long long incx, long long n, Out* result, cudaStream_t stream) {
  const int blocks = (int)std::min<long long>((n + 255) / 256, std::min(kLogdetMaxBlocks, 2 * h->num_sms));
  logdet_kernel<T, 256><<<blocks, 256, 0, stream>>>(x, incx, n, h->d_part, h->d_counter, h->d_logdet + 1);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  if constexpr (sizeof(Out) == sizeof(double)) {
    CUCHOL_CHECK(cudaMemcpyAsync(result, h->d_logdet + 1, sizeof(double), cudaMemcpyDeviceToHost, stream));
  } else {
    // narrow on the device so the host copy stays asynchronous
    narrow_double_kernel<<<1, 1, 0, stream>>>(h->d_logdet + 1, h->d_logdet_f);
    ++h->launches;
    CUCHOL_CHECK(cudaGetLastError());
    CUCHOL_CHECK(cudaMemcpyAsync(result, h->d_logdet_f, sizeof(float), cudaMemcpyDeviceToHost, stream));
  }
  return CUDA_SUCCESS;
}

}  // namespace


// ------------------------------------------------------------------------------
// Handle
// ------------------------------------------------------------------------------
namespace {

// Releases whatever a handle holds (any member may still be null).
void release_handle(CULAPACKhandle h) {
  if (h->s_panel != nullptr) cudaStreamSynchronize(h->s_panel);
  if (h->s_update != nullptr) cudaStreamSynchronize(h->s_update);
  cudaFree(h->ws);
  cudaFree(h->d_words);
  cudaFreeHost(h->h_words);
  cudaFree(h->d_logdet);
  cudaFree(h->d_logdet_f);
  cudaFreeHost(h->h_logdet);
  cudaFree(h->d_part);
  cudaFree(h->d_counter);
  cudaFree(h->desc_dev);
  cudaFreeHost(h->desc_host);
  if (h->ev_panel != nullptr) cudaEventDestroy(h->ev_panel);
  if (h->ev_update != nullptr) cudaEventDestroy(h->ev_update);
  if (h->s_panel != nullptr) cudaStreamDestroy(h->s_panel);
  if (h->s_update != nullptr) cudaStreamDestroy(h->s_update);
  delete h;
}

CUresult create_handle(CULAPACKhandle h);

}  // namespace

extern "C" CUCHOL_EXPORT CUresult cuLAPACKCreate(CULAPACKhandle* handle) {
  if (handle == nullptr) return CUDA_ERROR_INVALID_VALUE;
  auto* h = new (std::nothrow) __culapackhandle_st;
  if (h == nullptr) return CUDA_ERROR_OUT_OF_MEMORY;
  memset(h, 0, sizeof(*h));
  const CUresult rc = create_handle(h);
  if (rc != CUDA_SUCCESS) {
    release_handle(h);   // nothing of a failed creation is left behind
    return rc;
  }
  *handle = h;
  return CUDA_SUCCESS;
}

namespace {
CUresult create_handle(CULAPACKhandle h) {
  h->wait_limit = -1;
  CUCHOL_CHECK(cudaGetDevice(&h->device));
  {
    const char* e = getenv("CUCHOLESKY_FORCE_SIMT");   // testing: FP64 products on the SIMT engine
    h->force_simt = (e != nullptr && e[0] == '1') ? 1 : 0;
    const char* c = getenv("CUCHOLESKY_LAUUM_COLS");   // testing: ?lauum block-column width
    h->lauum_cols = (c != nullptr) ? std::max(0, atoi(c)) : 0;
  }
  {
    // a tuning file named by the environment replaces the built-in table once
    static std::once_flag once;
    std::call_once(once, [] {
      const char* path = getenv("CUCHOLESKY_TUNING");
      if (path != nullptr && path[0] != '\0' && !load_tuning(path))
        fprintf(stderr, "cucholesky: tuning file %s not loaded (unreadable or malformed)\n", path);
    });
  }
  CUCHOL_CHECK(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
  int lo = 0, hi = 0;
  CUCHOL_CHECK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  // blocking streams: they order after work the caller queued on the legacy stream.
  // The update stream sits between the panel stream and the lowest priority, which
  // is left for background work queued next to a factorization (the host-memory
  // ?potrf's updates of panels further right).
  const int mid = (hi < lo - 1) ? (lo + hi) / 2 : lo;
  CUCHOL_CHECK(cudaStreamCreateWithPriority(&h->s_panel, cudaStreamDefault, hi));
  CUCHOL_CHECK(cudaStreamCreateWithPriority(&h->s_update, cudaStreamDefault, mid));
  CUCHOL_CHECK(cudaEventCreateWithFlags(&h->ev_panel, cudaEventDisableTiming));
  CUCHOL_CHECK(cudaEventCreateWithFlags(&h->ev_update, cudaEventDisableTiming));
  CUCHOL_CHECK(dev_malloc(&h->d_words, 16 * sizeof(int)));
  CUCHOL_CHECK(cudaMemset(h->d_words, 0, 16 * sizeof(int)));
  CUCHOL_CHECK(cudaMallocHost(&h->h_words, 16 * sizeof(int)));
  CUCHOL_CHECK(dev_malloc(&h->d_logdet, 4 * sizeof(double)));
  CUCHOL_CHECK(dev_malloc(&h->d_logdet_f, 4 * sizeof(float)));
  CUCHOL_CHECK(cudaMallocHost(&h->h_logdet, 4 * sizeof(double)));
  CUCHOL_CHECK(dev_malloc(&h->d_part, kLogdetMaxBlocks * sizeof(double)));
  CUCHOL_CHECK(dev_malloc(&h->d_counter, sizeof(unsigned int)));
  CUCHOL_CHECK(cudaMemset(h->d_counter, 0, sizeof(unsigned int)));
  h->desc_bytes = size_t(8) << 20;
  CUCHOL_CHECK(dev_malloc(&h->desc_dev, h->desc_bytes));
  CUCHOL_CHECK(cudaMallocHost(&h->desc_host, h->desc_bytes));
  CUCHOL_CHECK(cudaDeviceSynchronize());
  return CUDA_SUCCESS;
}
}  // namespace

extern "C" CUCHOL_EXPORT CUresult cuLAPACKDestroy(CULAPACKhandle h) {
  if (h == nullptr) return CUDA_ERROR_INVALID_VALUE;
  CUCHOL_CHECK(cudaStreamSynchronize(h->s_panel));
  CUCHOL_CHECK(cudaStreamSynchronize(h->s_update));
  release_handle(h);
  return CUDA_SUCCESS;
}

// ---- testing hooks (include/cucholesky_ext.h) ---------------------------------------
extern "C" CUCHOL_EXPORT CUresult cuLAPACKFailAllocation(int after) {
  g_fail_after.store(after < 0 ? -1 : after);
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuLAPACKSetWaitLimit(CULAPACKhandle h, int iterations) {
  if (h == nullptr) return CUDA_ERROR_INVALID_VALUE;
  h->wait_limit = iterations;
  return CUDA_SUCCESS;
}

// ------------------------------------------------------------------------------
// C ABI.  Argument checks follow the reference drivers: lapack/dpotrf.c:173-179
// (potrf, -4), lapack/dtrtri.c:330-336 (trtri, -5), lapack/dlauum.c (-4),
// lapack/dpotri.c:29-35 (-4).  n == 0 returns at once.
// ------------------------------------------------------------------------------
namespace {

inline bool bad_uplo(CBlasUplo u) { return u != CBlasLower && u != CBlasUpper; }

template <typename T>
CUresult api_potrf(const char* name, CULAPACKhandle h, CBlasUplo uplo, size_t n, CUdeviceptr A, size_t lda,
                   long* info, double* logdet) {
  *info = 0;
  if (lda < n) *info = -4;
  if (*info != 0) {
    if (xerbla != nullptr) xerbla(name, -*info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (n == 0) {
    if (logdet) *logdet = 0.0;
    return CUDA_SUCCESS;
  }
  if (h == nullptr || bad_uplo(uplo) || n > (size_t)INT_MAX) return CUDA_ERROR_INVALID_VALUE;
  return potrf_run<T>(h, uplo == CBlasUpper, (int)n, reinterpret_cast<T*>(A), (long long)lda, info, logdet);
}

template <typename T>
CUresult api_trtri(const char* name, CULAPACKhandle h, CBlasUplo uplo, CBlasDiag diag, size_t n, CUdeviceptr A,
                   size_t lda, long* info) {
  *info = 0;
  if (lda < n) *info = -5;
  if (*info != 0) {
    if (xerbla != nullptr) xerbla(name, -*info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (n == 0) return CUDA_SUCCESS;
  if (h == nullptr || bad_uplo(uplo) || n > (size_t)INT_MAX) return CUDA_ERROR_INVALID_VALUE;
  return trtri_run<T>(h, uplo == CBlasUpper, diag == CBlasUnit, (int)n, reinterpret_cast<T*>(A), (long long)lda,
                      info);
}

template <typename T>
CUresult api_lauum(const char* name, CULAPACKhandle h, CBlasUplo uplo, size_t n, CUdeviceptr A, size_t lda,
                   long* info) {
  *info = 0;
  if (lda < n) *info = -4;
  if (*info != 0) {
    if (xerbla != nullptr) xerbla(name, -*info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (n == 0) return CUDA_SUCCESS;
  if (h == nullptr || bad_uplo(uplo) || n > (size_t)INT_MAX) return CUDA_ERROR_INVALID_VALUE;
  return lauum_run<T>(h, uplo == CBlasUpper, (int)n, reinterpret_cast<T*>(A), (long long)lda);
}

template <typename T>
CUresult api_potri(const char* name, CULAPACKhandle h, CBlasUplo uplo, size_t n, CUdeviceptr A, size_t lda,
                   long* info) {
  *info = 0;
  if (lda < n) *info = -4;
  if (*info != 0) {
    if (xerbla != nullptr) xerbla(name, -*info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (n == 0) return CUDA_SUCCESS;
  if (h == nullptr || bad_uplo(uplo) || n > (size_t)INT_MAX) return CUDA_ERROR_INVALID_VALUE;
  const bool up = (uplo == CBlasUpper);
  CUCHOL_CHECK_CU(trtri_run<T>(h, up, false, (int)n, reinterpret_cast<T*>(A), (long long)lda, info));
  if (*info != 0) return CUDA_SUCCESS;
  return lauum_run<T>(h, up, (int)n, reinterpret_cast<T*>(A), (long long)lda);
}

template <typename T>
CUresult api_trti22(CULAPACKhandle h, CBlasUplo uplo, CBlasDiag diag, size_t n, CUdeviceptr A, size_t lda,
                    CUdeviceptr B, size_t ldb, CUdeviceptr info, CUstream stream) {
  if (h == nullptr || bad_uplo(uplo) || lda < n || ldb < n) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0) return CUDA_SUCCESS;
  return trti22_run<T>(h, uplo == CBlasUpper, diag == CBlasUnit, (int)n, reinterpret_cast<const T*>(A),
                       (long long)lda, reinterpret_cast<T*>(B), (long long)ldb, reinterpret_cast<int*>(info),
                       reinterpret_cast<cudaStream_t>(stream));
}

template <typename T, typename Out>
CUresult api_logdet(CULAPACKhandle h, CUdeviceptr x, size_t incx, size_t n, Out* result, CUstream stream) {
  if (n == 0) {
    *result = Out(0);
    return CUDA_SUCCESS;
  }
  if (h == nullptr || result == nullptr) return CUDA_ERROR_INVALID_VALUE;
  return logdet_run<T, Out>(h, reinterpret_cast<const T*>(x), (long long)incx, (long long)n, result,
                            reinterpret_cast<cudaStream_t>(stream));
}

}  // namespace

#define CUCHOL_API_TYPE(P, T, R)                                                                          \
  extern "C" CUCHOL_EXPORT CUresult cu##P##potrf(CULAPACKhandle h, CBlasUplo u, size_t n, CUdeviceptr A, size_t lda,    \
                                   long* info) {                                                          \
    return api_potrf<T>("cu" #P "potrf", h, u, n, A, lda, info, nullptr);                                 \
  }                                                                                                       \
  extern "C" CUCHOL_EXPORT CUresult cu##P##trtri(CULAPACKhandle h, CBlasUplo u, CBlasDiag d, size_t n, CUdeviceptr A,   \
                                   size_t lda, long* info) {                                              \
    return api_trtri<T>("cu" #P "trtri", h, u, d, n, A, lda, info);                                       \
  }                                                                                                       \
  extern "C" CUCHOL_EXPORT CUresult cu##P##lauum(CULAPACKhandle h, CBlasUplo u, size_t n, CUdeviceptr A, size_t lda,    \
                                   long* info) {                                                          \
    return api_lauum<T>("cu" #P "lauum", h, u, n, A, lda, info);                                          \
  }                                                                                                       \
  extern "C" CUCHOL_EXPORT CUresult cu##P##potri(CULAPACKhandle h, CBlasUplo u, size_t n, CUdeviceptr A, size_t lda,    \
                                   long* info) {                                                          \
    return api_potri<T>("cu" #P "potri", h, u, n, A, lda, info);                                          \
  }                                                                                                       \
  extern "C" CUCHOL_EXPORT CUresult cu##P##trti22(CULAPACKhandle h, CBlasUplo u, CBlasDiag d, size_t n, CUdeviceptr A,  \
                                    size_t lda, CUdeviceptr B, size_t ldb, CUdeviceptr info, CUstream s) { \
    return api_trti22<T>(h, u, d, n, A, lda, B, ldb, info, s);                                            \
  }                                                                                                       \
  extern "C" CUCHOL_EXPORT CUresult cu##P##logdet(CULAPACKhandle h, CUdeviceptr x, size_t incx, size_t n, R* result,    \
                                    CUstream s) {                                                         \
    return api_logdet<T, R>(h, x, incx, n, result, s);                                                    \
  }

CUCHOL_API_TYPE(S, float, float)
CUCHOL_API_TYPE(D, double, double)
CUCHOL_API_TYPE(C, cuFloatComplex, float)
CUCHOL_API_TYPE(Z, cuDoubleComplex, double)

// ------------------------------------------------------------------------------
// Extensions (include/cucholesky_ext.h)
// ------------------------------------------------------------------------------
#define CUCHOL_API_LOGDET(P, T)                                                                            \
  extern "C" CUCHOL_EXPORT CUresult cu##P##potrfLogdet(CULAPACKhandle h, CBlasUplo u, size_t n, CUdeviceptr A, \
                                                       size_t lda, double* logdet, long* info) {           \
    double ld = 0.0;                                                                                       \
    CUresult r = api_potrf<T>("cu" #P "potrfLogdet", h, u, n, A, lda, info, &ld);                          \
    if (r == CUDA_SUCCESS && *info == 0 && logdet != nullptr) *logdet = ld;                                \
    return r;                                                                                              \
  }
CUCHOL_API_LOGDET(S, float)
CUCHOL_API_LOGDET(D, double)
CUCHOL_API_LOGDET(C, cuFloatComplex)
CUCHOL_API_LOGDET(Z, cuDoubleComplex)

extern "C" CUCHOL_EXPORT CUresult cuLAPACKGetLaunchCount(CULAPACKhandle h, unsigned long long* count) {
  if (h == nullptr || count == nullptr) return CUDA_ERROR_INVALID_VALUE;
  *count = h->launches;
  return CUDA_SUCCESS;
}

// ---- tuning table (tuning.cuh) -------------------------------------------------------
extern "C" CUCHOL_EXPORT CUresult cuLAPACKLoadTuning(const char* path) {
  if (path == nullptr) return CUDA_ERROR_INVALID_VALUE;
  return load_tuning(path) ? CUDA_SUCCESS : CUDA_ERROR_INVALID_VALUE;
}

extern "C" CUCHOL_EXPORT CUresult cuLAPACKSetPotrfBlocks(CULAPACKhandle h, int sub) {
  if (h == nullptr || sub < 0 || sub > kMaxSub) return CUDA_ERROR_INVALID_VALUE;
  h->potrf_sub = sub;
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuLAPACKGetPotrfBlocks(CULAPACKhandle h, char type, size_t n, int* sub) {
  if (sub == nullptr || strchr("SDCZ", type) == nullptr || type == '\0') return CUDA_ERROR_INVALID_VALUE;
  *sub = (h != nullptr && h->potrf_sub > 0) ? h->potrf_sub : tuned_potrf_sub(type, (long long)n);
  return CUDA_SUCCESS;
}

// ------------------------------------------------------------------------------
// BLAS layer (include/blas.h): cu?gemm2, cu?syrk, cu?herk on the same engines,
// queued on the caller's stream.  Argument checks follow blas/dgemm.c:154-171,
// blas/dsyrk.c:166-179 and blas/zherk.c:190-205.
// ------------------------------------------------------------------------------
struct __cublashandle_st {
  CULAPACKhandle lh;
};

extern "C" CUCHOL_EXPORT CUresult cuBLASCreate(CUBLAShandle* handle) {
  if (handle == nullptr) return CUDA_ERROR_INVALID_VALUE;
  auto* b = new (std::nothrow) __cublashandle_st;
  if (b == nullptr) return CUDA_ERROR_OUT_OF_MEMORY;
  CUresult r = cuLAPACKCreate(&b->lh);
  if (r != CUDA_SUCCESS) {
    delete b;
    return r;
  }
  *handle = b;
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuBLASDestroy(CUBLAShandle b) {
  if (b == nullptr) return CUDA_ERROR_INVALID_VALUE;
  CUresult r = cuLAPACKDestroy(b->lh);
  delete b;
  return r;
}

namespace {

template <typename T>
bool eq(const T& a, RealOf<T> r) {
  if constexpr (Traits<T>::complex) return a.x == r && a.y == 0;
  else return a == r;
}

// Operand view of op(X) as "rows x k" (rows_first) or "k x rows" (for B).
template <typename T>
void view_a(GemmProblem<T>& p, CBlasTranspose tr, CUdeviceptr A, size_t lda) {
  p.a = reinterpret_cast<const T*>(A);
  if (tr == CBlasNoTrans) { p.a_rs = 1; p.a_ks = (long long)lda; }
  else { p.a_rs = (long long)lda; p.a_ks = 1; p.conj_a = (tr == CBlasConjTrans); }
}
template <typename T>
void view_b(GemmProblem<T>& p, CBlasTranspose tr, CUdeviceptr B, size_t ldb) {
  p.b = reinterpret_cast<const T*>(B);
  if (tr == CBlasNoTrans) { p.b_rs = (long long)ldb; p.b_ks = 1; }
  else { p.b_rs = 1; p.b_ks = (long long)ldb; p.conj_b = (tr == CBlasConjTrans); }
}

inline bool bad_trans(CBlasTranspose t) { return t != CBlasNoTrans && t != CBlasTrans && t != CBlasConjTrans; }

template <typename T>
CUresult api_gemm2(const char* name, CUBLAShandle bh, CBlasTranspose ta, CBlasTranspose tb, size_t m, size_t n,
                   size_t k, T alpha, CUdeviceptr A, size_t lda, CUdeviceptr B, size_t ldb, T beta, CUdeviceptr C,
                   size_t ldc, CUdeviceptr D, size_t ldd, CUstream stream) {
  const size_t nRowA = (ta == CBlasNoTrans) ? m : k;
  const size_t nRowB = (tb == CBlasNoTrans) ? k : n;
  int info = 0;
  if (lda < nRowA) info = 8;
  else if (ldb < nRowB) info = 10;
  else if (ldc < m) info = 13;
  else if (ldd < m) info = 15;
  if (info != 0) {
    if (xerbla != nullptr) xerbla(name, info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (m == 0 || n == 0 || (C == D && ldc == ldd && (eq(alpha, 0) || k == 0) && eq(beta, 1))) return CUDA_SUCCESS;
  if (bh == nullptr || bad_trans(ta) || bad_trans(tb) || m > INT_MAX || n > INT_MAX || k > INT_MAX)
    return CUDA_ERROR_INVALID_VALUE;
  GemmProblem<T> p = problem<T>();
  view_a<T>(p, ta, A, lda);
  view_b<T>(p, tb, B, ldb);
  p.c = reinterpret_cast<T*>(D); p.c_rs = 1; p.c_cs = (long long)ldd;
  if (!eq(beta, 0)) { p.cin = reinterpret_cast<const T*>(C); p.cin_rs = 1; p.cin_cs = (long long)ldc; }
  p.alpha = alpha; p.beta = beta;
  p.m = (int)m; p.n = (int)n; p.k = (int)k;
  if (k == 0 || eq(alpha, 0)) { p.k = 0; }
  return gemm<T>(bh->lh, p, reinterpret_cast<cudaStream_t>(stream), nullptr);
}

// C := alpha op(A) op(A)^H + beta C on one triangle (herk: alpha, beta real; syrk: the
// transpose without conjugation).
template <typename T>
CUresult api_rankk(const char* name, bool herm, CUBLAShandle bh, CBlasUplo uplo, CBlasTranspose tr, size_t n,
                   size_t k, RealOf<T> alpha, CUdeviceptr A, size_t lda, RealOf<T> beta, CUdeviceptr C, size_t ldc,
                   CUstream stream) {
  const size_t nRowA = (tr == CBlasNoTrans) ? n : k;
  int info = 0;
  if (herm && tr == CBlasTrans) info = 2;
  else if (lda < nRowA) info = 7;
  else if (ldc < n) info = 10;
  if (info != 0) {
    if (xerbla != nullptr) xerbla(name, info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (n == 0 || ((alpha == 0 || k == 0) && beta == 1)) return CUDA_SUCCESS;
  if (bh == nullptr || bad_uplo(uplo) || bad_trans(tr) || n > INT_MAX || k > INT_MAX)
    return CUDA_ERROR_INVALID_VALUE;
  GemmProblem<T> p = problem<T>();
  const CBlasTranspose t2 = (tr == CBlasNoTrans) ? CBlasNoTrans : CBlasTrans;
  view_a<T>(p, t2, A, lda);
  p.b = p.a; p.b_rs = p.a_rs; p.b_ks = p.a_ks;
  if (herm) {
    // lower: A A^H (N) or A^H A (C); the upper triangle is the lower triangle of
    // the conjugate, read through the transposed view of C
    const bool cA = (tr != CBlasNoTrans);
    p.conj_a = cA; p.conj_b = !cA;
    if (uplo == CBlasUpper) { p.conj_a = !p.conj_a; p.conj_b = !p.conj_b; }
    p.real_diag = 1;
  }
  if (uplo == CBlasLower) { p.c_rs = 1; p.c_cs = (long long)ldc; }
  else { p.c_rs = (long long)ldc; p.c_cs = 1; }
  p.c = reinterpret_cast<T*>(C);
  if (beta != 0) { p.cin = p.c; p.cin_rs = p.c_rs; p.cin_cs = p.c_cs; }
  p.alpha = from_real<T>(alpha); p.beta = from_real<T>(beta);
  p.lower_only = 1;
  p.m = (int)n; p.n = (int)n; p.k = (alpha == 0) ? 0 : (int)k;
  return gemm<T>(bh->lh, p, reinterpret_cast<cudaStream_t>(stream), nullptr);
}

}  // namespace

#define CUCHOL_API_GEMM(P, T)                                                                                   \
  extern "C" CUCHOL_EXPORT CUresult cu##P##gemm2(CUBLAShandle h, CBlasTranspose ta, CBlasTranspose tb, size_t m, \
                                                 size_t n, size_t k, T alpha, CUdeviceptr A, size_t lda,        \
                                                 CUdeviceptr B, size_t ldb, T beta, CUdeviceptr C, size_t ldc,  \
                                                 CUdeviceptr D, size_t ldd, CUstream s) {                       \
    return api_gemm2<T>("cu" #P "gemm2", h, ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, D, ldd, s);  \
  }
CUCHOL_API_GEMM(S, float)
CUCHOL_API_GEMM(D, double)
CUCHOL_API_GEMM(C, cuFloatComplex)
CUCHOL_API_GEMM(Z, cuDoubleComplex)

#define CUCHOL_API_RANKK(NAME, T, HERM)                                                                         \
  extern "C" CUCHOL_EXPORT CUresult NAME(CUBLAShandle h, CBlasUplo u, CBlasTranspose tr, size_t n, size_t k,   \
                                         RealOf<T> alpha, CUdeviceptr A, size_t lda, RealOf<T> beta,            \
                                         CUdeviceptr C, size_t ldc, CUstream s) {                               \
    return api_rankk<T>(#NAME, HERM, h, u, tr, n, k, alpha, A, lda, beta, C, ldc, s);                          \
  }
CUCHOL_API_RANKK(cuSsyrk, float, false)
CUCHOL_API_RANKK(cuDsyrk, double, false)
CUCHOL_API_RANKK(cuCherk, cuFloatComplex, true)
CUCHOL_API_RANKK(cuZherk, cuDoubleComplex, true)

#include "blas3.cuh"
#include "batched.cuh"
#include "bpersist.cuh"
#include "mixed.cuh"
#include "ozaki_driver.cuh"
#include "hostmem.cuh"
#include "rng.cuh"
