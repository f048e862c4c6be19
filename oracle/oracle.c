/*
 * CPU restatement of the reference's dense SPD path (garymacindoe/cuda-cholesky):
 * ?POTRF, ?TRTRI, ?LAUUM, ?POTRI and ?LOGDET in s/d/c/z, column-major.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: the tests, the smoke
 * check and the bench's CPU-baseline leg call it to check or time against; the
 * product (the CUDA library) never links or calls it.
 *
 * Each routine restates the blocked algorithm of the reference source it cites,
 * with the same block sizes, loop order and failure rules, in plain C with the
 * BLAS3 pieces written as loops (OpenMP over independent columns).  It is pinned
 * against the reference library itself (oracle/_ref, built by oracle/ref.mk) and
 * against committed golden vectors by tests/test_oracle.py.
 *
 * One deliberate difference: ?logdet for double complex accumulates log(Re x) in
 * double.  The reference's zlogdet uses logf(crealf(x)) (lapack/zlogdet.c:18,22),
 * which loses double precision; the maths of the routine is the FP64 sum.
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <string.h>

typedef float complex cfloat;
typedef double complex cdouble;

static inline size_t mn(size_t a, size_t b) { return a < b ? a : b; }

/* Element access: column-major, A(i,j) = A[i + j*lda]. */
#define E(A, lda, i, j) (A)[(size_t)(i) + (size_t)(j) * (lda)]

/*
 * DEFINE_ORACLE(T, R, P, CJ, RE)
 *   T  element type, R its real type, P the routine prefix,
 *   CJ(x) complex conjugate (identity for real types), RE(x) real part.
 */
#define DEFINE_ORACLE(T, R, P, CJ, RE, SQRT)                                          \
                                                                                      \
/* Unblocked Cholesky of a diagonal block; reference lapack/dpotrf.c:34-81          \
 * (complex: lapack/zpotrf.c:35-84).  Upper is row-oriented (dot products),          \
 * lower is column-oriented (axpy updates), failure on a pivot <= 0 or NaN; the      \
 * upper branch stores the failing pivot back, the lower one does not. */            \
static void P##potf2(char uplo, size_t n, T *A, size_t lda, long *info) {            \
  if (uplo == 'U') {                                                                 \
    for (size_t i = 0; i < n; i++) {                                                 \
      R t = 0;                                                                       \
      for (size_t k = 0; k < i; k++) t += RE(E(A, lda, k, i) * CJ(E(A, lda, k, i))); \
      R aii = RE(E(A, lda, i, i)) - t;                                               \
      if (aii <= 0 || isnan(aii)) { E(A, lda, i, i) = aii; *info = (long)i + 1; return; } \
      aii = SQRT(aii);                                                               \
      E(A, lda, i, i) = aii;                                                         \
      for (size_t j = i + 1; j < n; j++) {                                           \
        T s = 0;                                                                     \
        for (size_t k = 0; k < i; k++) s += E(A, lda, k, j) * CJ(E(A, lda, k, i));   \
        E(A, lda, i, j) = (E(A, lda, i, j) - s) / aii;                               \
      }                                                                              \
    }                                                                                \
  } else {                                                                           \
    for (size_t j = 0; j < n; j++) {                                                 \
      for (size_t k = 0; k < j; k++) {                                               \
        T t = CJ(E(A, lda, j, k));                                                   \
        for (size_t i = j; i < n; i++) E(A, lda, i, j) -= t * E(A, lda, i, k);       \
      }                                                                              \
      R ajj = RE(E(A, lda, j, j));                                                   \
      if (ajj <= 0 || isnan(ajj)) { *info = (long)j + 1; return; }                   \
      ajj = SQRT(ajj);                                                               \
      E(A, lda, j, j) = ajj;                                                         \
      for (size_t i = j + 1; i < n; i++) E(A, lda, i, j) /= ajj;                     \
    }                                                                                \
  }                                                                                  \
}                                                                                    \
                                                                                     \
/* Blocked left-looking Cholesky; reference lapack/dpotrf.c:83-146 (nb 16 upper,     \
 * 32 lower, :97), each step: rank-k update of the diagonal block (dsyrk/zherk),     \
 * unblocked factor, panel update (dgemm) and panel solve (dtrsm). */                \
void orc_##P##potrf(char uplo, size_t n, T *A, size_t lda, long *info) {             \
  *info = 0;                                                                         \
  if (lda < n) { *info = -4; return; }                                               \
  if (n == 0) return;                                                                \
  const size_t nb = (uplo == 'U') ? 16 : 32;                                         \
  if (n < nb) { P##potf2(uplo, n, A, lda, info); return; }                           \
  if (uplo == 'U') {                                                                 \
    for (size_t j = 0; j < n; j += nb) {                                             \
      const size_t jb = mn(nb, n - j);                                               \
      /* A11 -= A01^H A01 (upper triangle) */                                        \
      for (size_t c = 0; c < jb; c++)                                                \
        for (size_t r = 0; r <= c; r++) {                                            \
          T s = 0;                                                                   \
          for (size_t k = 0; k < j; k++) s += CJ(E(A, lda, k, j + r)) * E(A, lda, k, j + c); \
          E(A, lda, j + r, j + c) -= s;                                              \
        }                                                                            \
      P##potf2('U', jb, &E(A, lda, j, j), lda, info);                                \
      if (*info) { *info += (long)j; return; }                                       \
      if (j + jb < n) {                                                              \
        const size_t m = n - j - jb;                                                 \
        /* A12 -= A01^H A02, then A12 := U11^-H A12 */                               \
        _Pragma("omp parallel for schedule(static)")                                 \
        for (size_t c = 0; c < m; c++) {                                             \
          T *col = &E(A, lda, 0, j + jb + c);                                        \
          for (size_t r = 0; r < jb; r++) {                                          \
            T s = 0;                                                                 \
            for (size_t k = 0; k < j; k++) s += CJ(E(A, lda, k, j + r)) * col[k];    \
            col[j + r] -= s;                                                         \
          }                                                                          \
          for (size_t r = 0; r < jb; r++) {                                          \
            T s = col[j + r];                                                        \
            for (size_t k = 0; k < r; k++) s -= CJ(E(A, lda, j + k, j + r)) * col[j + k]; \
            col[j + r] = s / CJ(E(A, lda, j + r, j + r));                            \
          }                                                                          \
        }                                                                            \
      }                                                                              \
    }                                                                                \
  } else {                                                                           \
    for (size_t j = 0; j < n; j += nb) {                                             \
      const size_t jb = mn(nb, n - j);                                               \
      /* A11 -= A10 A10^H (lower triangle) */                                        \
      for (size_t c = 0; c < jb; c++)                                                \
        for (size_t k = 0; k < j; k++) {                                             \
          T t = CJ(E(A, lda, j + c, k));                                             \
          for (size_t r = c; r < jb; r++) E(A, lda, j + r, j + c) -= E(A, lda, j + r, k) * t; \
        }                                                                            \
      P##potf2('L', jb, &E(A, lda, j, j), lda, info);                                \
      if (*info) { *info += (long)j; return; }                                       \
      if (j + jb < n) {                                                              \
        const size_t m = n - j - jb;                                                 \
        /* A21 -= A20 A10^H, then A21 := A21 L11^-H */                               \
        _Pragma("omp parallel for schedule(static)")                                 \
        for (size_t r0 = 0; r0 < m; r0 += 64) {                                      \
          const size_t re = mn(m, r0 + 64);                                          \
          for (size_t c = 0; c < jb; c++) {                                          \
            T *dst = &E(A, lda, j + jb, j + c);                                      \
            for (size_t k = 0; k < j; k++) {                                         \
              T t = CJ(E(A, lda, j + c, k));                                         \
              const T *src = &E(A, lda, j + jb, k);                                  \
              for (size_t r = r0; r < re; r++) dst[r] -= src[r] * t;                 \
            }                                                                        \
          }                                                                          \
          for (size_t c = 0; c < jb; c++) {                                          \
            T *dst = &E(A, lda, j + jb, j + c);                                      \
            for (size_t k = 0; k < c; k++) {                                         \
              T t = CJ(E(A, lda, j + c, j + k));                                     \
              const T *src = &E(A, lda, j + jb, j + k);                              \
              for (size_t r = r0; r < re; r++) dst[r] -= src[r] * t;                 \
            }                                                                        \
            T d = CJ(E(A, lda, j + c, j + c));                                       \
            for (size_t r = r0; r < re; r++) dst[r] /= d;                            \
          }                                                                          \
        }                                                                            \
      }                                                                              \
    }                                                                                \
  }                                                                                  \
}                                                                                    \
                                                                                     \
/* Unblocked triangular inverse; reference lapack/dtrtri.c:43-96.  Upper scans      \
 * columns forward, lower scans them backward; info = first zero pivot met. */       \
static void P##trti2(char uplo, char diag, size_t n, T *A, size_t lda, long *info) { \
  const int nonunit = (diag != 'U');                                                 \
  if (n == 0) return;                                                                \
  if (uplo == 'U') {                                                                 \
    for (size_t j = 0; j < n; j++) {                                                 \
      T ajj;                                                                         \
      if (nonunit) {                                                                 \
        if (E(A, lda, j, j) == (T)0) { *info = (long)j + 1; return; }                \
        E(A, lda, j, j) = (T)1 / E(A, lda, j, j);                                    \
        ajj = -E(A, lda, j, j);                                                      \
      } else ajj = -1;                                                               \
      for (size_t k = 0; k < j; k++) {                                               \
        T t = E(A, lda, k, j);                                                       \
        if (nonunit) E(A, lda, k, j) *= E(A, lda, k, k);                             \
        for (size_t i = 0; i < k; i++) E(A, lda, i, j) += t * E(A, lda, i, k);       \
      }                                                                              \
      for (size_t i = 0; i < j; i++) E(A, lda, i, j) *= ajj;                         \
    }                                                                                \
  } else {                                                                           \
    size_t j = n - 1;                                                                \
    do {                                                                             \
      T ajj;                                                                         \
      if (nonunit) {                                                                 \
        if (E(A, lda, j, j) == (T)0) { *info = (long)j + 1; return; }                \
        E(A, lda, j, j) = (T)1 / E(A, lda, j, j);                                    \
        ajj = -E(A, lda, j, j);                                                      \
      } else ajj = -1;                                                               \
      for (size_t i = n - 1; i > j; i--) {                                           \
        T t = E(A, lda, i, j);                                                       \
        if (nonunit) E(A, lda, i, j) *= E(A, lda, i, i);                             \
        for (size_t k = i + 1; k < n; k++) E(A, lda, k, j) += t * E(A, lda, k, i);   \
      }                                                                              \
      for (size_t i = j + 1; i < n; i++) E(A, lda, i, j) *= ajj;                     \
    } while (j-- > 0);                                                               \
  }                                                                                  \
}                                                                                    \
                                                                                     \
/* Blocked in-place triangular inverse; reference lapack/dtrtri.c:98-164 (nb 64).   \
 * Upper walks block columns forward: A01 := T00 A01 (dtrmm), A01 := -A01 A11^-1     \
 * (dtrsm), invert A11.  Lower walks them backward with the mirrored steps. */       \
void orc_##P##trtri(char uplo, char diag, size_t n, T *A, size_t lda, long *info) {  \
  *info = 0;                                                                         \
  if (lda < n) { *info = -5; return; }                                               \
  if (n == 0) return;                                                                \
  const size_t nb = 64;                                                              \
  const int nonunit = (diag != 'U');                                                 \
  if (n < nb) { P##trti2(uplo, diag, n, A, lda, info); return; }                     \
  if (uplo == 'U') {                                                                 \
    for (size_t j = 0; j < n; j += nb) {                                             \
      const size_t jb = mn(nb, n - j);                                               \
      _Pragma("omp parallel for schedule(static)")                                   \
      for (size_t c = 0; c < jb; c++) {                                              \
        T *col = &E(A, lda, 0, j + c);                                               \
        /* col[0:j] := T00 col[0:j], T00 upper (already inverted) */                 \
        for (size_t i = 0; i < j; i++) {                                             \
          T s = nonunit ? E(A, lda, i, i) * col[i] : col[i];                         \
          for (size_t k = i + 1; k < j; k++) s += E(A, lda, i, k) * col[k];          \
          col[i] = s;                                                                \
        }                                                                            \
      }                                                                              \
      /* A01 := -A01 A11^-1, A11 upper: solve X A11 = -A01 column by column */       \
      _Pragma("omp parallel for schedule(static)")                                   \
      for (size_t r0 = 0; r0 < j; r0 += 64) {                                        \
        const size_t re = mn(j, r0 + 64);                                            \
        for (size_t c = 0; c < jb; c++) {                                            \
          T *dst = &E(A, lda, 0, j + c);                                             \
          for (size_t r = r0; r < re; r++) dst[r] = -dst[r];                         \
          for (size_t k = 0; k < c; k++) {                                           \
            T t = E(A, lda, j + k, j + c);                                           \
            const T *src = &E(A, lda, 0, j + k);                                     \
            for (size_t r = r0; r < re; r++) dst[r] -= src[r] * t;                   \
          }                                                                          \
          if (nonunit) { T d = E(A, lda, j + c, j + c);                              \
            for (size_t r = r0; r < re; r++) dst[r] /= d; }                          \
        }                                                                            \
      }                                                                              \
      P##trti2('U', diag, jb, &E(A, lda, j, j), lda, info);                          \
      if (*info) { *info += (long)j; return; }                                       \
    }                                                                                \
  } else {                                                                           \
    size_t j = (n + nb - 1) / nb * nb;                                               \
    do {                                                                             \
      j -= nb;                                                                       \
      const size_t jb = mn(nb, n - j);                                               \
      if (j + jb < n) {                                                              \
        const size_t m = n - j - jb;                                                 \
        _Pragma("omp parallel for schedule(static)")                                 \
        for (size_t c = 0; c < jb; c++) {                                            \
          T *col = &E(A, lda, j + jb, j + c);                                        \
          /* col := T22 col, T22 lower (already inverted), bottom-up */              \
          for (size_t ii = m; ii-- > 0;) {                                           \
            T s = nonunit ? E(A, lda, j + jb + ii, j + jb + ii) * col[ii] : col[ii]; \
            for (size_t k = 0; k < ii; k++) s += E(A, lda, j + jb + ii, j + jb + k) * col[k]; \
            col[ii] = s;                                                             \
          }                                                                          \
        }                                                                            \
        /* A21 := -A21 A11^-1, A11 lower: columns from the last one back */          \
        _Pragma("omp parallel for schedule(static)")                                 \
        for (size_t r0 = 0; r0 < m; r0 += 64) {                                      \
          const size_t re = mn(m, r0 + 64);                                          \
          for (size_t c = jb; c-- > 0;) {                                            \
            T *dst = &E(A, lda, j + jb, j + c);                                      \
            for (size_t r = r0; r < re; r++) dst[r] = -dst[r];                       \
            for (size_t k = c + 1; k < jb; k++) {                                    \
              T t = E(A, lda, j + k, j + c);                                         \
              const T *src = &E(A, lda, j + jb, j + k);                              \
              for (size_t r = r0; r < re; r++) dst[r] -= src[r] * t;                 \
            }                                                                        \
            if (nonunit) { T d = E(A, lda, j + c, j + c);                            \
              for (size_t r = r0; r < re; r++) dst[r] /= d; }                        \
          }                                                                          \
        }                                                                            \
      }                                                                              \
      P##trti2('L', diag, jb, &E(A, lda, j, j), lda, info);                          \
      if (*info) { *info += (long)j; return; }                                       \
    } while (j > 0);                                                                 \
  }                                                                                  \
}                                                                                    \
                                                                                     \
/* Unblocked U U^H / L^H L; reference lapack/dlauum.c:43-69 (zlauum.c:44-70). */     \
static void P##lauu2(char uplo, size_t n, T *A, size_t lda) {                        \
  if (uplo == 'U') {                                                                 \
    for (size_t j = 0; j < n; j++) {                                                 \
      T ajj = CJ(E(A, lda, j, j));                                                   \
      for (size_t i = 0; i <= j; i++) E(A, lda, i, j) *= ajj;                        \
      for (size_t k = j + 1; k < n; k++) {                                           \
        T t = CJ(E(A, lda, j, k));                                                   \
        for (size_t i = 0; i <= j; i++) E(A, lda, i, j) += t * E(A, lda, i, k);      \
      }                                                                              \
    }                                                                                \
  } else {                                                                           \
    for (size_t j = 0; j < n; j++)                                                   \
      for (size_t i = j; i < n; i++) {                                               \
        E(A, lda, i, j) *= CJ(E(A, lda, i, i));                                      \
        for (size_t k = i + 1; k < n; k++) E(A, lda, i, j) += CJ(E(A, lda, k, i)) * E(A, lda, k, j); \
      }                                                                              \
  }                                                                                  \
}                                                                                    \
                                                                                     \
/* Blocked U U^H (upper) or L^H L (lower); reference lapack/dlauum.c:71-129          \
 * (nb 16 upper, 32 lower): dtrmm with the diagonal block, unblocked product of      \
 * the block, then the dgemm and dsyrk/zherk contributions of the trailing rows. */  \
void orc_##P##lauum(char uplo, size_t n, T *A, size_t lda, long *info) {             \
  *info = 0;                                                                         \
  if (lda < n) { *info = -4; return; }                                               \
  if (n == 0) return;                                                                \
  const size_t nb = (uplo == 'U') ? 16 : 32;                                         \
  if (nb > n) { P##lauu2(uplo, n, A, lda); return; }                                 \
  if (uplo == 'U') {                                                                 \
    for (size_t i = 0; i < n; i += nb) {                                             \
      const size_t ib = mn(nb, n - i);                                               \
      /* A01 := A01 U11^H, then A11 := U11 U11^H, then A01 += A02 A12^H and         \
         A11 += A12 A12^H */                                                         \
      _Pragma("omp parallel for schedule(static)")                                   \
      for (size_t r = 0; r < i; r++) {                                               \
        T row[64], acc[64];                                                          \
        for (size_t c = 0; c < ib; c++) row[c] = E(A, lda, r, i + c);                \
        for (size_t c = 0; c < ib; c++) {                                            \
          T s = 0;                                                                   \
          for (size_t k = c; k < ib; k++) s += row[k] * CJ(E(A, lda, i + c, i + k)); \
          acc[c] = s;                                                                \
        }                                                                            \
        for (size_t c = 0; c < ib; c++) {                                            \
          T s = acc[c];                                                              \
          for (size_t k = i + ib; k < n; k++) s += E(A, lda, r, k) * CJ(E(A, lda, i + c, k)); \
          E(A, lda, r, i + c) = s;                                                   \
        }                                                                            \
      }                                                                              \
      P##lauu2('U', ib, &E(A, lda, i, i), lda);                                      \
      for (size_t c = 0; c < ib; c++)                                                \
        for (size_t r = 0; r <= c; r++) {                                            \
          T s = 0;                                                                   \
          for (size_t k = i + ib; k < n; k++) s += E(A, lda, i + r, k) * CJ(E(A, lda, i + c, k)); \
          E(A, lda, i + r, i + c) += s;                                              \
        }                                                                            \
    }                                                                                \
  } else {                                                                           \
    for (size_t i = 0; i < n; i += nb) {                                             \
      const size_t ib = mn(nb, n - i);                                               \
      /* A10 := L11^H A10, A11 := L11^H L11, A10 += A21^H A20, A11 += A21^H A21 */   \
      _Pragma("omp parallel for schedule(static)")                                   \
      for (size_t c = 0; c < i; c++) {                                               \
        T col[64], acc[64];                                                          \
        for (size_t r = 0; r < ib; r++) col[r] = E(A, lda, i + r, c);                \
        for (size_t r = 0; r < ib; r++) {                                            \
          T s = 0;                                                                   \
          for (size_t k = r; k < ib; k++) s += CJ(E(A, lda, i + k, i + r)) * col[k]; \
          acc[r] = s;                                                                \
        }                                                                            \
        for (size_t r = 0; r < ib; r++) {                                            \
          T s = acc[r];                                                              \
          for (size_t k = i + ib; k < n; k++) s += CJ(E(A, lda, k, i + r)) * E(A, lda, k, c); \
          E(A, lda, i + r, c) = s;                                                   \
        }                                                                            \
      }                                                                              \
      P##lauu2('L', ib, &E(A, lda, i, i), lda);                                      \
      for (size_t c = 0; c < ib; c++)                                                \
        for (size_t r = c; r < ib; r++) {                                            \
          T s = 0;                                                                   \
          for (size_t k = i + ib; k < n; k++) s += CJ(E(A, lda, k, i + r)) * E(A, lda, k, i + c); \
          E(A, lda, i + r, i + c) += s;                                              \
        }                                                                            \
    }                                                                                \
  }                                                                                  \
}                                                                                    \
                                                                                     \
/* Inverse from the Cholesky factor; reference lapack/dpotri.c:4-23. */              \
void orc_##P##potri(char uplo, size_t n, T *A, size_t lda, long *info) {             \
  *info = 0;                                                                         \
  if (lda < n) { *info = -4; return; }                                               \
  if (n == 0) return;                                                                \
  orc_##P##trtri(uplo, 'N', n, A, lda, info);                                        \
  if (*info) return;                                                                 \
  orc_##P##lauum(uplo, n, A, lda, info);                                             \
}                                                                                    \
                                                                                     \
/* 2 * sum log(Re x[i*incx]); reference lapack/dlogdet.c:10-25.  Accumulates in     \
 * double for every type (the reference accumulates s/c in float). */                \
double orc_##P##logdet(const T *x, size_t incx, size_t n) {                          \
  double total = 0.0;                                                                \
  for (size_t i = 0; i < n; i++) total += log((double)RE(x[i * incx]));              \
  return 2.0 * total;                                                                \
}

#define ID(x) (x)
#define REAL_RE(x) (x)
DEFINE_ORACLE(float, float, s, ID, REAL_RE, sqrtf)
DEFINE_ORACLE(double, double, d, ID, REAL_RE, sqrt)
DEFINE_ORACLE(cfloat, float, c, conjf, crealf, sqrtf)
DEFINE_ORACLE(cdouble, double, z, conj, creal, sqrt)
