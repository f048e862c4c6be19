// Triangular BLAS3 entry points of include/blas.h on the same engines (included at the
// end of lapack.cu):
//   cu?trmm2  X := alpha op(A) B  or  alpha B op(A), out of place
//             (reference blas/dtrmm.c:374, include/blas.h:214-232): one product on the
//             GEMM engine with the triangular operand masked (unit diagonal implicit).
//   cu?trsm   B := alpha op(A)^-1 B  or  alpha B op(A)^-1, in place
//             (reference blas/dtrsm.c:218, include/blas.h:235-253): blocked substitution
//             with inverted 128-wide diagonal blocks; each block step is two products
//             (W = inv(T_II) B_I, then the remaining rows -= T(rest, I) W) and a copy of
//             W back into B.  Right-side solves are left-side solves of the transposed
//             views (X op(A) = B  <=>  op(A)^T X^T = B^T).
// Argument checks and XERBLA positions follow blas/dtrsm.c:223-233.

namespace {

// The logical view of a triangular operand T = op(A): T(i, k) = t[i * rs + k * cs],
// conjugated if conj, nonzero only in its lower (or upper) triangle.
template <typename T>
struct TriView {
  const T* t;
  long long rs, cs;
  bool conj, lower, unit;
};

template <typename T>
TriView<T> tri_view(CBlasUplo uplo, CBlasTranspose tr, CBlasDiag diag, const T* A, long long lda) {
  TriView<T> v;
  v.t = A;
  v.unit = (diag == CBlasUnit);
  if (tr == CBlasNoTrans) {
    v.rs = 1; v.cs = lda; v.conj = false; v.lower = (uplo == CBlasLower);
  } else {
    v.rs = lda; v.cs = 1; v.conj = (tr == CBlasConjTrans); v.lower = (uplo == CBlasUpper);
  }
  return v;
}

// B := alpha B on a view (alpha_zero: B := 0, as BLAS does, whatever B holds)
template <typename T>
__global__ void scale_view_kernel(T* __restrict__ b, long long rs, long long cs, int m, int n, T alpha,
                                  int alpha_zero) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)m * n) return;
  const int i = (int)(e % m), j = (int)(e / m);
  T& x = b[i * rs + j * cs];
  x = alpha_zero ? zero<T>() : mul(alpha, x);
}

// B (view m x n, strides brs, bcs) := inv(T) B with T the m x m triangular view v.
template <typename T>
CUresult trsm_left(CULAPACKhandle h, const TriView<T>& v, int m, int n, T* B, long long brs, long long bcs,
                   cudaStream_t s) {
  constexpr int nb = Tune<T>::nb;
  using Smem = DiagSmem<T, nb>;
  const int nblk = (m + nb - 1) / nb;
  const long long ldw = (long long)round_up((size_t)nb, 2);
  // workspace: the inverted diagonal blocks (nb x nb each, column-major, in the
  // orientation of the view), then W (nb x n)
  const size_t dbytes = round_up(sizeof(T) * (size_t)nblk * nb * nb, 256);
  const size_t need = dbytes + sizeof(T) * (size_t)ldw * n;
  // growing the workspace frees the old one: work still queued on the caller's
  // stream may use it
  if (need > h->ws_bytes) CUCHOL_CHECK(cudaStreamSynchronize(s));
  CUCHOL_CHECK_CU(ensure_workspace(h, need));
  T* Dinv = static_cast<T*>(h->ws);
  T* W = reinterpret_cast<T*>(static_cast<char*>(h->ws) + dbytes);
  CUCHOL_CHECK_CU(set_smem<T>((const void*)diag_invert_kernel<T, nb, kDiagThreads2>, Smem::bytes));
  for (int I = 0; I < nblk; ++I) {
    const int r0 = I * nb, rb = std::min(nb, m - r0);
    T* D = Dinv + (size_t)I * nb * nb;
    // D(i, k) = T(r0 + i, r0 + k) (no conjugation yet), then invert its triangle in
    // place through the lower view of that triangle
    CUCHOL_CHECK_CU(copy_view<T>(h, v.t + r0 * v.rs + r0 * v.cs, v.rs, v.cs, D, 1, nb, rb, rb, false, s, nullptr));
    const long long lrs = v.lower ? 1 : nb, lcs = v.lower ? nb : 1;
    diag_invert_kernel<T, nb, kDiagThreads2><<<1, kDiagThreads2, Smem::bytes, s>>>(D, lrs, lcs, rb, nb,
                                                                                   v.unit ? 1 : 0);
    ++h->launches;
    CUCHOL_CHECK(cudaGetLastError());
  }
  for (int q = 0; q < nblk; ++q) {
    const int I = v.lower ? q : nblk - 1 - q;     // forward for lower, backward for upper
    const int r0 = I * nb, rb = std::min(nb, m - r0);
    const T* D = Dinv + (size_t)I * nb * nb;
    // W = inv(T_II) B_I
    GemmProblem<T> p1 = problem<T>();
    p1.a = D; p1.a_rs = 1; p1.a_ks = nb; p1.conj_a = v.conj;
    p1.tri_a = v.lower ? TRI_LOWER : TRI_UPPER;
    p1.unit_a = v.unit;   // the unit diagonal stays implicit in the inverse too
    p1.b = B + r0 * brs; p1.b_rs = bcs; p1.b_ks = brs;
    p1.c = W; p1.c_rs = 1; p1.c_cs = ldw;
    p1.m = rb; p1.n = n; p1.k = rb;
    CUCHOL_CHECK_CU(gemm<T>(h, p1, s, nullptr));
    // the rows still to solve -= T(rows, I) W
    const int lo = v.lower ? r0 + rb : 0, hi = v.lower ? m : r0;
    if (hi > lo) {
      GemmProblem<T> p2 = problem<T>();
      p2.a = v.t + lo * v.rs + r0 * v.cs; p2.a_rs = v.rs; p2.a_ks = v.cs; p2.conj_a = v.conj;
      p2.b = W; p2.b_rs = ldw; p2.b_ks = 1;
      p2.c = B + lo * brs; p2.c_rs = brs; p2.c_cs = bcs;
      p2.cin = p2.c; p2.cin_rs = brs; p2.cin_cs = bcs;
      p2.alpha = from_real<T>(RealOf<T>(-1)); p2.beta = from_real<T>(RealOf<T>(1));
      p2.m = hi - lo; p2.n = n; p2.k = rb;
      CUCHOL_CHECK_CU(gemm<T>(h, p2, s, nullptr));
    }
    CUCHOL_CHECK_CU(copy_view<T>(h, W, 1, ldw, B + r0 * brs, brs, bcs, rb, n, false, s, nullptr));
  }
  return CUDA_SUCCESS;
}

inline bool bad_side(CBlasSide s) { return s != CBlasLeft && s != CBlasRight; }
inline bool bad_diag(CBlasDiag d) { return d != CBlasUnit && d != CBlasNonUnit; }

template <typename T>
CUresult api_trsm(const char* name, CUBLAShandle bh, CBlasSide side, CBlasUplo uplo, CBlasTranspose tr,
                  CBlasDiag diag, size_t m, size_t n, T alpha, CUdeviceptr A, size_t lda, CUdeviceptr B,
                  size_t ldb, CUstream stream) {
  const size_t nRowA = (side == CBlasLeft) ? m : n;
  int info = 0;
  if (lda < nRowA) info = 9;
  else if (ldb < m) info = 11;
  if (info != 0) {
    if (xerbla != nullptr) xerbla(name, info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (m == 0 || n == 0) return CUDA_SUCCESS;
  if (bh == nullptr || bad_side(side) || bad_uplo(uplo) || bad_trans(tr) || bad_diag(diag) || m > INT_MAX ||
      n > INT_MAX)
    return CUDA_ERROR_INVALID_VALUE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  T* Bp = reinterpret_cast<T*>(B);
  const T* Ap = reinterpret_cast<const T*>(A);
  // logical problem: inv(T) X-view, T = op(A) (left) or op(A)^T (right, on B^T)
  long long brs = 1, bcs = (long long)ldb;
  int mm = (int)m, nn = (int)n;
  TriView<T> v;
  if (side == CBlasLeft) {
    v = tri_view<T>(uplo, tr, diag, Ap, (long long)lda);
  } else {
    // X op(A) = B  <=>  op(A)^T X^T = B^T: the transpose of op(A) is A (tr = T),
    // A^T (tr = N) or conj(A) (tr = C)
    const CBlasTranspose t2 = (tr == CBlasNoTrans) ? CBlasTrans : CBlasNoTrans;
    v = tri_view<T>(uplo, t2, diag, Ap, (long long)lda);
    v.conj = (tr == CBlasConjTrans);
    brs = (long long)ldb; bcs = 1;
    mm = (int)n; nn = (int)m;
  }
  if (!eq(alpha, 1)) {
    const long long tot = (long long)mm * nn;
    scale_view_kernel<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(Bp, brs, bcs, mm, nn, alpha,
                                                                       eq(alpha, 0) ? 1 : 0);
    ++bh->lh->launches;
    CUCHOL_CHECK(cudaGetLastError());
    if (eq(alpha, 0)) return CUDA_SUCCESS;
  }
  return trsm_left<T>(bh->lh, v, mm, nn, Bp, brs, bcs, s);
}

template <typename T>
CUresult api_trmm2(const char* name, CUBLAShandle bh, CBlasSide side, CBlasUplo uplo, CBlasTranspose tr,
                   CBlasDiag diag, size_t m, size_t n, T alpha, CUdeviceptr A, size_t lda, CUdeviceptr B,
                   size_t ldb, CUdeviceptr X, size_t ldx, CUstream stream) {
  const size_t nRowA = (side == CBlasLeft) ? m : n;
  int info = 0;
  if (lda < nRowA) info = 9;
  else if (ldb < m) info = 11;
  else if (ldx < m) info = 13;
  if (info != 0) {
    if (xerbla != nullptr) xerbla(name, info);
    return CUDA_ERROR_INVALID_VALUE;
  }
  if (m == 0 || n == 0) return CUDA_SUCCESS;
  if (bh == nullptr || bad_side(side) || bad_uplo(uplo) || bad_trans(tr) || bad_diag(diag) || m > INT_MAX ||
      n > INT_MAX)
    return CUDA_ERROR_INVALID_VALUE;
  const T* Ap = reinterpret_cast<const T*>(A);
  const T* Bp = reinterpret_cast<const T*>(B);
  GemmProblem<T> p = problem<T>();
  const TriView<T> v = tri_view<T>(uplo, tr, diag, Ap, (long long)lda);
  if (side == CBlasLeft) {
    // X(i, j) = sum_k T(i, k) B(k, j)
    p.a = v.t; p.a_rs = v.rs; p.a_ks = v.cs; p.conj_a = v.conj;
    p.tri_a = v.lower ? TRI_LOWER : TRI_UPPER; p.unit_a = v.unit;
    p.b = Bp; p.b_rs = (long long)ldb; p.b_ks = 1;
    p.k = (int)m;
  } else {
    // X(i, j) = sum_k B(i, k) T(k, j): the B operand of the engine is T^T
    p.a = Bp; p.a_rs = 1; p.a_ks = (long long)ldb;
    p.b = v.t; p.b_rs = v.cs; p.b_ks = v.rs; p.conj_b = v.conj;
    p.tri_b = v.lower ? TRI_UPPER : TRI_LOWER; p.unit_b = v.unit;
    p.k = (int)n;
  }
  p.c = reinterpret_cast<T*>(X); p.c_rs = 1; p.c_cs = (long long)ldx;
  p.alpha = alpha;
  p.m = (int)m; p.n = (int)n;
  if (eq(alpha, 0)) p.k = 0;
  return gemm<T>(bh->lh, p, reinterpret_cast<cudaStream_t>(stream), nullptr);
}

}  // namespace

#define CUCHOL_API_TRI(P, T)                                                                                     \
  extern "C" CUCHOL_EXPORT CUresult cu##P##trsm(CUBLAShandle h, CBlasSide side, CBlasUplo u, CBlasTranspose tr,   \
                                                CBlasDiag d, size_t m, size_t n, T alpha, CUdeviceptr A,          \
                                                size_t lda, CUdeviceptr B, size_t ldb, CUstream s) {              \
    return api_trsm<T>("cu" #P "trsm", h, side, u, tr, d, m, n, alpha, A, lda, B, ldb, s);                       \
  }                                                                                                              \
  extern "C" CUCHOL_EXPORT CUresult cu##P##trmm2(CUBLAShandle h, CBlasSide side, CBlasUplo u, CBlasTranspose tr,  \
                                                 CBlasDiag d, size_t m, size_t n, T alpha, CUdeviceptr A,         \
                                                 size_t lda, CUdeviceptr B, size_t ldb, CUdeviceptr X,            \
                                                 size_t ldx, CUstream s) {                                        \
    return api_trmm2<T>("cu" #P "trmm2", h, side, u, tr, d, m, n, alpha, A, lda, B, ldb, X, ldx, s);             \
  }
CUCHOL_API_TRI(S, float)
CUCHOL_API_TRI(D, double)
CUCHOL_API_TRI(C, cuFloatComplex)
CUCHOL_API_TRI(Z, cuDoubleComplex)
