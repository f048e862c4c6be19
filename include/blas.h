/*
 * cucholesky-b200: drop-in C API for the GPU BLAS3 layer under the dense SPD path
 * (reference include/blas.h), implemented by libcucholesky.so on the same sm_100a
 * engines as the LAPACK routines: FP64 tensor-core (DMMA) tiles with TMA-staged
 * operands for double, a SIMT engine for the other types.
 *
 * Prototypes are those of the reference's include/blas.h (line numbers cited per
 * entry).  Complex scalars are passed by value as in the reference (C99
 * `float complex` / `double complex`; in C++ the layout-identical cuFloatComplex /
 * cuDoubleComplex).  Argument errors: XERBLA(position) and
 * CUDA_ERROR_INVALID_VALUE, as in blas/dgemm.c:156-168.  Calls are queued on the
 * caller's stream and return without waiting.
 */
#ifndef CUCHOLESKY_BLAS_H
#define CUCHOLESKY_BLAS_H

#include <stddef.h>
#include <cuda.h>
#ifdef __cplusplus
#include <cuComplex.h>
typedef cuFloatComplex cucholesky_cfloat;
typedef cuDoubleComplex cucholesky_cdouble;
#else
typedef float _Complex cucholesky_cfloat;
typedef double _Complex cucholesky_cdouble;
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* BLAS enums, castable to char (reference include/blas.h:24-27). */
#ifndef CUCHOLESKY_NO_CBLAS_ENUMS
typedef enum { CBlasNoTrans = 'N', CBlasTrans = 'T', CBlasConjTrans = 'C' } CBlasTranspose;
typedef enum { CBlasLower = 'L', CBlasUpper = 'U' } CBlasUplo;
typedef enum { CBlasLeft = 'L', CBlasRight = 'R' } CBlasSide;
typedef enum { CBlasNonUnit = 'N', CBlasUnit = 'U' } CBlasDiag;
#endif

/* Argument-error hook (reference include/blas.h:39-44, blas/xerbla.c:9).  Called
 * with the routine name and the 1-based position of the bad argument; may be set
 * to NULL or replaced by the caller. */
typedef void (*xerbla_t)(const char *, long);
extern xerbla_t xerbla;

/* CUDA error hook (reference include/error.h:23-32, multigpu/error.c:11). */
typedef void (*errorHandler_t)(const char *, const char *, const char *, int,
                               int, const char * (*)(int));
extern errorHandler_t errorHandler;

/* BLAS handle (reference include/blas.h:152-154, blas/handle.c:84-95). */
typedef struct __cublashandle_st * CUBLAShandle;
CUresult cuBLASCreate(CUBLAShandle *);
CUresult cuBLASDestroy(CUBLAShandle);

/* Rank-k update of one triangle: C := alpha op(A) op(A)^T + beta C
 * (reference include/blas.h:157-166, blas/dsyrk.c:163). */
CUresult cuSsyrk(CUBLAShandle, CBlasUplo, CBlasTranspose, size_t, size_t,
                 float, CUdeviceptr, size_t, float, CUdeviceptr, size_t, CUstream);
CUresult cuDsyrk(CUBLAShandle, CBlasUplo, CBlasTranspose, size_t, size_t,
                 double, CUdeviceptr, size_t, double, CUdeviceptr, size_t, CUstream);

/* Hermitian rank-k update: C := alpha op(A) op(A)^H + beta C, op = N or C
 * (reference include/blas.h:168-177, blas/zherk.c:190). */
CUresult cuCherk(CUBLAShandle, CBlasUplo, CBlasTranspose, size_t, size_t,
                 float, CUdeviceptr, size_t, float, CUdeviceptr, size_t, CUstream);
CUresult cuZherk(CUBLAShandle, CBlasUplo, CBlasTranspose, size_t, size_t,
                 double, CUdeviceptr, size_t, double, CUdeviceptr, size_t, CUstream);

/* Out-of-place matrix multiply D := alpha op(A) op(B) + beta C, and the in-place
 * macros (reference include/blas.h:179-215, blas/dgemm.c:148). */
#define cuSgemm(h, tA, tB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream) \
        cuSgemm2(h, tA, tB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, C, ldc, stream)
#define cuDgemm(h, tA, tB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream) \
        cuDgemm2(h, tA, tB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, C, ldc, stream)
#define cuCgemm(h, tA, tB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream) \
        cuCgemm2(h, tA, tB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, C, ldc, stream)
#define cuZgemm(h, tA, tB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, stream) \
        cuZgemm2(h, tA, tB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, C, ldc, stream)
CUresult cuSgemm2(CUBLAShandle, CBlasTranspose, CBlasTranspose, size_t, size_t, size_t,
                  float, CUdeviceptr, size_t, CUdeviceptr, size_t,
                  float, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);
CUresult cuDgemm2(CUBLAShandle, CBlasTranspose, CBlasTranspose, size_t, size_t, size_t,
                  double, CUdeviceptr, size_t, CUdeviceptr, size_t,
                  double, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);
CUresult cuCgemm2(CUBLAShandle, CBlasTranspose, CBlasTranspose, size_t, size_t, size_t,
                  cucholesky_cfloat, CUdeviceptr, size_t, CUdeviceptr, size_t,
                  cucholesky_cfloat, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);
CUresult cuZgemm2(CUBLAShandle, CBlasTranspose, CBlasTranspose, size_t, size_t, size_t,
                  cucholesky_cdouble, CUdeviceptr, size_t, CUdeviceptr, size_t,
                  cucholesky_cdouble, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);

/* Out-of-place triangular matrix multiply X := alpha op(A) B (side L) or alpha B op(A)
 * (side R), A triangular (uplo, diag) (reference include/blas.h:214-232,
 * blas/dtrmm.c:374). */
CUresult cuStrmm2(CUBLAShandle, CBlasSide, CBlasUplo, CBlasTranspose, CBlasDiag, size_t, size_t,
                  float, CUdeviceptr, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);
CUresult cuDtrmm2(CUBLAShandle, CBlasSide, CBlasUplo, CBlasTranspose, CBlasDiag, size_t, size_t,
                  double, CUdeviceptr, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);
CUresult cuCtrmm2(CUBLAShandle, CBlasSide, CBlasUplo, CBlasTranspose, CBlasDiag, size_t, size_t,
                  cucholesky_cfloat, CUdeviceptr, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);
CUresult cuZtrmm2(CUBLAShandle, CBlasSide, CBlasUplo, CBlasTranspose, CBlasDiag, size_t, size_t,
                  cucholesky_cdouble, CUdeviceptr, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);

/* Triangular solve in place: B := alpha op(A)^-1 B (side L) or alpha B op(A)^-1
 * (side R) (reference include/blas.h:235-253, blas/dtrsm.c:218). */
CUresult cuStrsm(CUBLAShandle, CBlasSide, CBlasUplo, CBlasTranspose, CBlasDiag, size_t, size_t,
                 float, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);
CUresult cuDtrsm(CUBLAShandle, CBlasSide, CBlasUplo, CBlasTranspose, CBlasDiag, size_t, size_t,
                 double, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);
CUresult cuCtrsm(CUBLAShandle, CBlasSide, CBlasUplo, CBlasTranspose, CBlasDiag, size_t, size_t,
                 cucholesky_cfloat, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);
CUresult cuZtrsm(CUBLAShandle, CBlasSide, CBlasUplo, CBlasTranspose, CBlasDiag, size_t, size_t,
                 cucholesky_cdouble, CUdeviceptr, size_t, CUdeviceptr, size_t, CUstream);

#ifdef __cplusplus
}
#endif

#endif
