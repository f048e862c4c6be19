// FP64 Cholesky factor with Ozaki-sliced trailing updates (included at the end of
// lapack.cu; uses its launch helpers).  No counterpart in the reference library: it
// is ?potrf (lapack/dpotrf.c:172) with the trailing SYRK of every outer block done by
// the INT8 tensor-core emulation of ozaki.cuh instead of the FP64 DMMA engine.
//
// Schedule: the ?potrf schedule (nb = 128, outer blocks of sub x 128 columns as sub
// sub-panels, sub from the tuning table: 8 below n = 49152, 16 from there on;
// lookahead depth 1, two streams).  After the sub-panels of an outer
// block the panel rows below it (the packed buffer P) are cut into S slices
// (slice_kernel, ping-pong buffers); the lookahead update of the next outer block
// (panel stream) and the rest of the trailing matrix (update stream) both run on
// update_kernel from those slices, with k = the outer block: the two epilogues per tile
// (FP64 read-modify-write of C) are paid once per outer block, so a wide block makes
// the INT8 products dominate.  The updates inside the outer block (each
// sub-panel's on the ones after it, k = 128) stay on the DMMA engine.
#include "ozaki.cuh"

namespace {

CUresult ozaki_update(CULAPACKhandle h, const int8_t* sl, int R, int S, long long kp, int k, const int* expo,
                      int a0, int b0, double* c, long long crs, long long ccs, int m, int ncols, cudaStream_t s,
                      const int* stop) {
  if (m <= 0 || ncols <= 0) return CUDA_SUCCESS;
  EncodeTiledFn fn = encode_tiled();
  if (fn == nullptr) return CUDA_ERROR_NOT_SUPPORTED;
  CUtensorMap map;
  const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)S * R};
  const cuuint64_t strides[1] = {(cuuint64_t)kp};
  const cuuint32_t box[2] = {128, (cuuint32_t)oz::BM}, es[2] = {1, 1};
  if (fn(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(sl), dims, strides, box, es,
         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return CUDA_ERROR_INVALID_VALUE;
  oz::Params q{};
  q.c = c; q.crs = crs; q.ccs = ccs;
  q.m = m; q.n = ncols; q.k = k; q.slices = S;
  q.a_row0 = a0; q.b_row0 = b0; q.expo = expo;
  q.tiles_m = (m + oz::BM - 1) / oz::BM;
  q.tiles_n = (ncols + oz::BN - 1) / oz::BN;
  q.err = h->d_words + 3;
  int tiles = 0;
  for (int r = 0; r < q.tiles_m; ++r) tiles += std::min(q.tiles_n, (r * oz::BM + oz::BM - 1) / oz::BN + 1);
  static bool attr = false;
  if (!attr) {
    CUCHOL_CHECK(cudaFuncSetAttribute(oz::update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      oz::SMEM_BYTES));
    attr = true;
  }
  oz::update_kernel<<<tiles, oz::THREADS, oz::SMEM_BYTES, s>>>(map, map, q, R, stop);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

CUresult potrf_ozaki_run(CULAPACKhandle h, bool upper, int n, double* A, long long lda, int S, long* info) {
  constexpr int nb = 128;
  const int NB = (h->potrf_sub > 0 ? h->potrf_sub : tuned_sub(TUNE_OZAKI, 'D', n)) * nb;
  using Smem = DiagSmem<double, nb>;
  const long long rs = upper ? lda : 1, cs = upper ? 1 : lda;
  auto at = [&](long long i, long long j) { return A + i * rs + j * cs; };
  cudaStream_t sp = h->s_panel, su = h->s_update;
  int* d_info = h->d_words;
  const long long ldp = (long long)round_up((size_t)n, 2);
  const long long kp = NB;                                   // slice row pitch (bytes)
  const size_t pbytes = round_up(sizeof(double) * 2 * (size_t)ldp * NB, 256);
  const size_t sbytes = round_up((size_t)S * n * kp, 256), ebytes = round_up(sizeof(int) * (size_t)n, 256);
  CUCHOL_CHECK_CU(ensure_workspace(h, pbytes + 2 * (sbytes + ebytes)));
  char* ws = static_cast<char*>(h->ws);
  double* pbuf[2] = {reinterpret_cast<double*>(ws), reinterpret_cast<double*>(ws) + (size_t)ldp * NB};
  int8_t* sbuf[2] = {reinterpret_cast<int8_t*>(ws + pbytes), reinterpret_cast<int8_t*>(ws + pbytes + sbytes)};
  int* ebuf[2] = {reinterpret_cast<int*>(ws + pbytes + 2 * sbytes),
                  reinterpret_cast<int*>(ws + pbytes + 2 * sbytes + ebytes)};

  CUCHOL_CHECK_CU(set_smem<double>((const void*)diag_factor_kernel<double, nb, kDiagThreads2>, Smem::bytes));
  CUCHOL_CHECK_CU(set_smem<double>((const void*)trsm_rows_kernel<double, double, double, double, OUT_CONVERT>,
                                   trsm_rows_smem<double>()));
  CUCHOL_CHECK(cudaMemsetAsync(d_info, 0, sizeof(int), sp));
  CUCHOL_CHECK(cudaMemsetAsync(h->d_logdet, 0, sizeof(double), sp));
  CUCHOL_CHECK(cudaEventRecord(h->ev_panel, sp));
  CUCHOL_CHECK(cudaStreamWaitEvent(su, h->ev_panel, 0));
  CUCHOL_CHECK(cudaEventRecord(h->ev_update, su));

  for (int j = 0, step = 0; j < n; j += NB, ++step) {
    const int jB = std::min(NB, n - j);
    const int m = n - j - jB;
    double* P = pbuf[step & 1];
    for (int s0 = 0; s0 < jB; s0 += nb) {
      const int c = j + s0, jb = std::min(nb, j + jB - c);
      const int mr = n - c - jb;
      diag_factor_kernel<double, nb, kDiagThreads2><<<1, kDiagThreads2, Smem::bytes, sp>>>(
          at(c, c), rs, cs, jb, nullptr, nb, c, d_info, h->d_logdet);
      ++h->launches;
      CUCHOL_CHECK(cudaGetLastError());
      if (mr == 0) break;
      double* Ps = P + s0 + (long long)s0 * ldp;   // P(r, .) = rows from j + nb
      trsm_rows_kernel<double, double, double, double, OUT_CONVERT><<<(mr + 63) / 64, 256, trsm_rows_smem<double>(), sp>>>(
          at(c + jb, c), rs, cs, mr, jb, at(c, c), rs, cs, Ps, 1, ldp, d_info, nullptr);
      ++h->launches;
      CUCHOL_CHECK(cudaGetLastError());
      if (s0 + nb < jB) {   // the outer block's remaining sub-panel columns by this one (DMMA)
        GemmProblem<double> u = problem<double>();
        u.a = Ps; u.a_rs = 1; u.a_ks = ldp;
        u.b = Ps; u.b_rs = 1; u.b_ks = ldp;
        u.c = at(c + nb, c + nb); u.c_rs = rs; u.c_cs = cs;
        u.cin = u.c; u.cin_rs = rs; u.cin_cs = cs;
        u.alpha = -1.0; u.beta = 1.0;
        u.lower_only = 1;
        u.m = n - c - nb; u.n = jB - s0 - nb; u.k = nb;
        CUCHOL_CHECK_CU(gemm<double>(h, u, sp, d_info));
      }
    }
    if (m == 0) break;
    // slices of the panel rows from j + NB (P rows NB - nb ..), k = jB
    int8_t* sl = sbuf[step & 1];
    int* ex = ebuf[step & 1];
    oz::slice_kernel<<<(m + 31) / 32, 256, 0, sp>>>(P + (NB - nb), 1, ldp, m, jB, S, sl, kp, ex, d_info);
    ++h->launches;
    CUCHOL_CHECK(cudaGetLastError());
    CUCHOL_CHECK(cudaEventRecord(h->ev_panel, sp));
    const int jB2 = std::min(NB, m);
    CUCHOL_CHECK(cudaStreamWaitEvent(sp, h->ev_update, 0));
    CUCHOL_CHECK_CU(ozaki_update(h, sl, m, S, kp, jB, ex, 0, 0, at(j + NB, j + NB), rs, cs, m, jB2, sp, d_info));
    CUCHOL_CHECK(cudaStreamWaitEvent(su, h->ev_panel, 0));
    if (m > jB2)
      CUCHOL_CHECK_CU(ozaki_update(h, sl, m, S, kp, jB, ex, jB2, jB2, at(j + NB + jB2, j + NB + jB2), rs, cs,
                                   m - jB2, m - jB2, su, d_info));
    CUCHOL_CHECK(cudaEventRecord(h->ev_update, su));
  }
  CUCHOL_CHECK(cudaEventRecord(h->ev_update, su));
  CUCHOL_CHECK(cudaStreamWaitEvent(sp, h->ev_update, 0));
  CUCHOL_CHECK(cudaMemcpyAsync(h->h_words, d_info, 4 * sizeof(int), cudaMemcpyDeviceToHost, sp));
  CUCHOL_CHECK(cudaStreamSynchronize(sp));
  CUCHOL_CHECK_CU(check_engine(h));
  *info = h->h_words[0];
  return CUDA_SUCCESS;
}

}  // namespace

// cu?potrf contract (argument errors, info, in place); slices in [4, 8].  slices = 0
// picks 8 below n = 8192 and 7 from there on: the products dropped by 7 slices are
// below 2^-56 k |P_i| |P_j| per update, far under the FP64 bound 10 n eps once n is
// large, for 28 instead of 36 slice products.
extern "C" CUCHOL_EXPORT CUresult cuDpotrfOzaki(CULAPACKhandle h, CBlasUplo uplo, size_t n, CUdeviceptr A,
                                                size_t lda, int slices, long* info) {
  if (info == nullptr) return CUDA_ERROR_INVALID_VALUE;
  *info = 0;
  if (slices == 0) slices = (n >= 8192) ? 7 : oz::MAX_SLICES;
  if (bad_uplo(uplo)) *info = -2;
  else if (lda < std::max<size_t>(1, n)) *info = -5;
  else if (slices < 4 || slices > oz::MAX_SLICES) *info = -6;
  if (*info != 0) {
    if (xerbla != nullptr) xerbla("cuDpotrfOzaki", -*info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (h == nullptr || n > (size_t)INT_MAX) return CUDA_ERROR_INVALID_VALUE;
  if (n == 0) return CUDA_SUCCESS;
  return potrf_ozaki_run(h, uplo == CBlasUpper, (int)n, reinterpret_cast<double*>(A), (long long)lda, slices, info);
}
