/*
 * cucholesky-b200: drop-in C API for the dense SPD path of the reference LAPACK
 * layer (?POTRF, ?TRTRI, ?TRTI22, ?LAUUM, ?POTRI, ?LOGDET on the GPU), implemented
 * by libcucholesky.so with hand-written sm_100a kernels.
 *
 * Every prototype below is identical to the one in the reference's
 * include/lapack.h (line numbers cited per entry), so code written against the
 * reference's GPU routines, and against its host-memory cuMultiGPU* routines,
 * links against this library unchanged.  The reference's CPU routines
 * (spotrf ... zpotri, ?logdet) are not exported by this library.
 *
 * Conventions kept from the reference:
 *   - column-major storage, only the `uplo` triangle is read or written;
 *   - CUdeviceptr matrices, host `long *info`;
 *   - argument errors: *info = -position, XERBLA(position) through the `xerbla`
 *     hook, return CUDA_ERROR_INVALID_VALUE (lapack/dpotrf.c:173-179);
 *   - numerical failure: CUDA_SUCCESS with *info = k > 0 (k = first non-positive
 *     or NaN leading minor for ?potrf, first zero pivot in the reference's scan
 *     order for ?trtri);
 *   - CUDA errors are passed to the `errorHandler` hook and returned
 *     (include/error.h:42-51).
 * Differences (documented, not observable through `info`):
 *   - *info is final when ?potrf/?trtri/?lauum/?potri return (the call waits for
 *     its own work); the reference returned with work possibly still queued.
 *   - the factor of a failing ?potrf is correct in its leading (info-1) x (info-1)
 *     part only, as in the reference; a singular ?trtri leaves A unmodified.
 */
#ifndef CUCHOLESKY_LAPACK_H
#define CUCHOLESKY_LAPACK_H

#include "blas.h"
#include "cumultigpu.h"

#ifdef __cplusplus
#define CUCHOLESKY_RESTRICT __restrict__
#else
#define CUCHOLESKY_RESTRICT restrict
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Handle: binds the device current at creation, owns streams, events and cached
 * device workspace (reference include/lapack.h:63-65, lapack/handle.c:77-88).
 * Not thread-safe; calls on one handle must not overlap. */
typedef struct __culapackhandle_st * CULAPACKhandle;
CUresult cuLAPACKCreate(CULAPACKhandle *);                              /* lapack.h:64 */
CUresult cuLAPACKDestroy(CULAPACKhandle);                               /* lapack.h:65 */

/* Cholesky factor A = L L^H (lower) or U^H U (upper), in place
 * (reference include/lapack.h:68-74, lapack/dpotrf.c:172). */
CUresult cuSpotrf(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);
CUresult cuDpotrf(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);
CUresult cuCpotrf(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);
CUresult cuZpotrf(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);

/* In-place triangular inverse (reference include/lapack.h:77-83, lapack/dtrtri.c:326). */
CUresult cuStrtri(CULAPACKhandle, CBlasUplo, CBlasDiag, size_t, CUdeviceptr, size_t, long *);
CUresult cuDtrtri(CULAPACKhandle, CBlasUplo, CBlasDiag, size_t, CUdeviceptr, size_t, long *);
CUresult cuCtrtri(CULAPACKhandle, CBlasUplo, CBlasDiag, size_t, CUdeviceptr, size_t, long *);
CUresult cuZtrtri(CULAPACKhandle, CBlasUplo, CBlasDiag, size_t, CUdeviceptr, size_t, long *);

/* Unblocked triangular inverse of one small block, B := A^-1, on a caller stream
 * with a device `int` info word (reference include/lapack.h:85-97,
 * lapack/dtrtri.c:301-324).  The reference accepts n <= 32; this library accepts
 * n <= 128 (n <= 64 for the double complex routine) and returns
 * CUDA_ERROR_INVALID_VALUE above that, as the reference does above 32. */
#define cuStrti2(handle, uplo, diag, n, A, lda, info) cuStrti22(handle, uplo, diag, n, A, lda, A, lda, info)
#define cuDtrti2(handle, uplo, diag, n, A, lda, info) cuDtrti22(handle, uplo, diag, n, A, lda, A, lda, info)
#define cuCtrti2(handle, uplo, diag, n, A, lda, info) cuCtrti22(handle, uplo, diag, n, A, lda, A, lda, info)
#define cuZtrti2(handle, uplo, diag, n, A, lda, info) cuZtrti22(handle, uplo, diag, n, A, lda, A, lda, info)
CUresult cuStrti22(CULAPACKhandle, CBlasUplo, CBlasDiag, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, CUdeviceptr, CUstream);
CUresult cuDtrti22(CULAPACKhandle, CBlasUplo, CBlasDiag, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, CUdeviceptr, CUstream);
CUresult cuCtrti22(CULAPACKhandle, CBlasUplo, CBlasDiag, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, CUdeviceptr, CUstream);
CUresult cuZtrti22(CULAPACKhandle, CBlasUplo, CBlasDiag, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, CUdeviceptr, CUstream);

/* U U^H (upper) or L^H L (lower) of a triangular factor, in place
 * (reference include/lapack.h:100-106, lapack/dlauum.c:154). */
CUresult cuSlauum(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);
CUresult cuDlauum(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);
CUresult cuClauum(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);
CUresult cuZlauum(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);

/* Inverse of A from its Cholesky factor: ?trtri then ?lauum
 * (reference include/lapack.h:109-115, lapack/dpotri.c:25-46). */
CUresult cuSpotri(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);
CUresult cuDpotri(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);
CUresult cuCpotri(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);
CUresult cuZpotri(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, long *);

/* 2 * sum_i log(Re x[i*incx]) (log det A when x is the factor's diagonal, incx =
 * lda + 1), queued on `stream`; *result is valid once the stream has synchronised
 * (reference include/lapack.h:166-169, lapack/dlogdet.c:37-74).  The sum is taken
 * in double for every type (the reference's ?logdet for single complex and
 * double complex take logf of the real part). */
CUresult cuSlogdet(CULAPACKhandle, CUdeviceptr, size_t, size_t,  float *, CUstream);
CUresult cuDlogdet(CULAPACKhandle, CUdeviceptr, size_t, size_t, double *, CUstream);
CUresult cuClogdet(CULAPACKhandle, CUdeviceptr, size_t, size_t,  float *, CUstream);
CUresult cuZlogdet(CULAPACKhandle, CUdeviceptr, size_t, size_t, double *, CUstream);

/* Host-memory routines (reference include/lapack.h:117-158).  A is a host array
 * (pageable or page-locked; a device or managed pointer also works); the call
 * copies the `uplo` triangle to the first device of the handle's CUmultiGPU, runs
 * the single-GPU routine there and copies the triangle back before it returns.
 * With page-locked A, cu?potrf copies each block column of the factor back while
 * the rest of the factorization runs.  Same argument checks as the reference
 * (lda < n: info -4, -5 for ?trtri); numerical failure (info > 0) returns
 * CUDA_ERROR_INVALID_VALUE as the reference's host-memory routines do
 * (lapack/dpotrf.c:330, lapack/dtrtri.c:499, lapack/dpotri.c:64), and a singular
 * ?trtri leaves A unmodified.  The handle caches one device buffer of the largest
 * matrix seen; calls on one handle must not overlap. */
typedef struct __cumultigpulapackhandle_st * CUmultiGPULAPACKhandle;
CUresult cuMultiGPULAPACKCreate(CUmultiGPULAPACKhandle *, CUmultiGPU);   /* lapack.h:120 */
CUresult cuMultiGPULAPACKDestroy(CUmultiGPULAPACKhandle);                /* lapack.h:121 */
CUresult cuMultiGPULAPACKSynchronize(CUmultiGPULAPACKhandle);            /* lapack.h:122 */

/* Cholesky factor in host memory (reference include/lapack.h:124-131, lapack/dpotrf.c:298). */
CUresult cuMultiGPUSpotrf(CUmultiGPULAPACKhandle, CBlasUplo, size_t, float * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUDpotrf(CUmultiGPULAPACKhandle, CBlasUplo, size_t, double * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUCpotrf(CUmultiGPULAPACKhandle, CBlasUplo, size_t, cucholesky_cfloat * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUZpotrf(CUmultiGPULAPACKhandle, CBlasUplo, size_t, cucholesky_cdouble * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);

/* Triangular inverse in host memory (reference include/lapack.h:133-140, lapack/dtrtri.c:470). */
CUresult cuMultiGPUStrtri(CUmultiGPULAPACKhandle, CBlasUplo, CBlasDiag, size_t, float * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUDtrtri(CUmultiGPULAPACKhandle, CBlasUplo, CBlasDiag, size_t, double * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUCtrtri(CUmultiGPULAPACKhandle, CBlasUplo, CBlasDiag, size_t, cucholesky_cfloat * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUZtrtri(CUmultiGPULAPACKhandle, CBlasUplo, CBlasDiag, size_t, cucholesky_cdouble * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);

/* Triangular square in host memory (reference include/lapack.h:142-149, lapack/dlauum.c:294). */
CUresult cuMultiGPUSlauum(CUmultiGPULAPACKhandle, CBlasUplo, size_t, float * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUDlauum(CUmultiGPULAPACKhandle, CBlasUplo, size_t, double * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUClauum(CUmultiGPULAPACKhandle, CBlasUplo, size_t, cucholesky_cfloat * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUZlauum(CUmultiGPULAPACKhandle, CBlasUplo, size_t, cucholesky_cdouble * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);

/* Inverse from the Cholesky factor in host memory (reference include/lapack.h:151-158, lapack/dpotri.c:48). */
CUresult cuMultiGPUSpotri(CUmultiGPULAPACKhandle, CBlasUplo, size_t, float * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUDpotri(CUmultiGPULAPACKhandle, CBlasUplo, size_t, double * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUCpotri(CUmultiGPULAPACKhandle, CBlasUplo, size_t, cucholesky_cfloat * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);
CUresult cuMultiGPUZpotri(CUmultiGPULAPACKhandle, CBlasUplo, size_t, cucholesky_cdouble * CUCHOLESKY_RESTRICT, size_t, long * CUCHOLESKY_RESTRICT);

#ifdef __cplusplus
}
#endif

#endif
