/*
 * Extensions of libcucholesky.so beyond the reference API.  Same conventions as
 * include/lapack.h (handle first, CUresult return, host `long *info`).  None of
 * these has a counterpart in the reference library.
 */
#ifndef CUCHOLESKY_EXT_H
#define CUCHOLESKY_EXT_H

#include "lapack.h"
#include "curng.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ?potrf that also returns log det A = 2 sum log L(j,j), accumulated by the
 * diagonal-block kernels as each block is factored (no second pass over the
 * diagonal).  *logdet is set only when *info == 0. */
CUresult cuDpotrfLogdet(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, double *, long *);
CUresult cuZpotrfLogdet(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, double *, long *);
CUresult cuSpotrfLogdet(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, double *, long *);
CUresult cuCpotrfLogdet(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, double *, long *);

/* Number of kernels this handle has launched since it was created (for
 * measurement; counts this library's own kernels only). */
CUresult cuLAPACKGetLaunchCount(CULAPACKhandle, unsigned long long *);

/* Tuning table (the counterpart of the reference's build-time include/config.h,
 * written by its blas/config.c): process-wide rows "potrf <S|D|C|Z> <n_min> <sub>"
 * choosing ?potrf's outer block (sub diagonal blocks of 128 columns, 64 for Z) for
 * orders n >= n_min.  Built-in rows were measured on a B200; cuLAPACKLoadTuning
 * replaces them with a file in the text format written by
 * cuda-cholesky_b200/cucholesky/tune.py (first line "cucholesky-tuning 1"; the
 * CUCHOLESKY_TUNING environment variable names one to load when the first handle is
 * created).  A malformed file leaves the table unchanged and returns
 * CUDA_ERROR_INVALID_VALUE.  Rows "ozaki D <n_min> <sub>" do the same for
 * cuDpotrfOzaki.  cuLAPACKSetPotrfBlocks overrides the table for one handle's ?potrf
 * and cuDpotrfOzaki (1..16; 0 restores the table); cuLAPACKGetPotrfBlocks reports the
 * value ?potrf of that type and order would use (handle may be NULL: the table alone). */
CUresult cuLAPACKLoadTuning(const char *);
CUresult cuLAPACKSetPotrfBlocks(CULAPACKhandle, int);
CUresult cuLAPACKGetPotrfBlocks(CULAPACKhandle, char, size_t, int *);

/* Batched factor, log det and inverse of many small SPD matrices of uneven sizes
 * (each matrix b: order n[b], device pointer A[b], leading dimension lda[b], all
 * in the same `uplo` storage).  No counterpart in the reference library.
 *
 * A plan records its whole sequence once into a CUDA graph, in one of two forms:
 *   nb = 8..64 (a multiple of 8): all matrices advance one nb-wide block column per
 *     step, and each step is a few grouped launches over the batch (diagonal blocks,
 *     panel solves, trailing updates), followed, with CUCHOL_BATCHED_POTRI, by the
 *     grouped inverse;
 *   nb = -1 (FP64 only): one persistent kernel; each CTA takes whole matrices from a
 *     queue ordered by size, largest first, and factors, log-dets and inverts each in
 *     place with 64 x 64 tile products on the FP64 tensor cores.
 * nb = 0 lets the plan pick by timing the candidates (grouped with nb 32 and 64, and
 * the persistent kernel for FP64) on an identity batch of the same shapes.  The plan
 * keeps the pointers: run it again after refilling the same buffers.
 * cuCholBatchedGetBlockSize reports the chosen nb (-1: the persistent kernel).
 *   cu?cholBatchedCreate  build (and tune) the plan; allocates its workspace
 *   cuCholBatchedRun      one graph launch on `stream`
 *   cuCholBatchedResults  waits, then copies info[b] (as ?potrf / ?potri) and
 *                         log det A_b (with CUCHOL_BATCHED_LOGDET) to the host */
typedef struct __cucholbatched_st * CUcholBatched;
#define CUCHOL_BATCHED_POTRF  1
#define CUCHOL_BATCHED_LOGDET 2
#define CUCHOL_BATCHED_POTRI  4
CUresult cuDcholBatchedCreate(CUcholBatched *, CULAPACKhandle, CBlasUplo, int, const int *, const CUdeviceptr *,
                              const int *, int, int);
CUresult cuScholBatchedCreate(CUcholBatched *, CULAPACKhandle, CBlasUplo, int, const int *, const CUdeviceptr *,
                              const int *, int, int);
CUresult cuCholBatchedRun(CUcholBatched, CUstream);
CUresult cuCholBatchedResults(CUcholBatched, long *, double *);
CUresult cuCholBatchedGetBlockSize(CUcholBatched, int *);
CUresult cuCholBatchedDestroy(CUcholBatched);

/* log det from a strided FP64 diagonal, 2 * sum_i log(x[i*incx]), for callers that
 * cannot allocate device memory.  No counterpart in the reference library.
 *
 * Who needs it: cuDlogdet keeps its scratch in a handle that cuLAPACKCreate
 * allocates with cudaMalloc (and the reference's cuDlogdet allocates and frees
 * on every call).  Some callers may not do that: code whose device memory is owned
 * by another allocator (a framework's caching allocator or a pool reserved at
 * start-up, where a cudaMalloc outside it fails or fragments the budget), and
 * loops that must not allocate or free after start-up because cudaFree can
 * synchronise the whole device.  This entry point takes no handle and calls no
 * cudaMalloc, cudaFree or other allocating routine: its scratch is a static device
 * array of about 32 KB that every GPU loading the library holds until exit.
 *
 * Limit: n <= 8,388,608 (the array holds one partial sum per 2048 elements);
 * larger n calls XERBLA with position 3 and returns CUDA_ERROR_INVALID_VALUE.
 * The work is queued on `stream`; *result is valid once the stream has
 * synchronised.  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current, and so does the first
 * call after the device's context was re-created (cudaDeviceReset): make that
 * first call before any stream capture.  Under lazy module loading (CUDA's
 * default) that first call can also make the driver load this library's kernels,
 * which takes device memory once; make it at start-up, or set
 * CUDA_MODULE_LOADING=EAGER.  All calls share the one array and each call clears
 * what must start at zero: calls that overlap on the GPU race. */
CUresult cuDlogdetNoAlloc(CUdeviceptr x, size_t incx, size_t n, double *result, CUstream stream);


/* Testing hooks for the failure paths (no counterpart in the reference library,
 * whose failure reporting is the CUresult of each call plus the errorHandler
 * callback, include/error.h:42-65 and multigpu/error.c:4-11).  Neither is needed in
 * normal use.
 *   cuLAPACKFailAllocation   after `after` more device allocations by this library
 *                            have succeeded, the next one fails as if the device
 *                            were out of memory (no cudaMalloc is attempted for it),
 *                            once: the routine that asked returns
 *                            CUDA_ERROR_OUT_OF_MEMORY through errorHandler, frees
 *                            what it had allocated, and its handle stays usable.
 *                            after < 0 clears a pending failure.
 *   cuLAPACKSetWaitLimit     the ticket-ordered triangular solves of cu?potrs poll a
 *                            counter that earlier blocks raise; a wait gives up after
 *                            `iterations` polls (< 0: the default, seconds), and the
 *                            call then returns CUDA_ERROR_LAUNCH_TIMEOUT through
 *                            errorHandler.  0 makes every such wait give up at once. */
CUresult cuLAPACKFailAllocation(int after);
CUresult cuLAPACKSetWaitLimit(CULAPACKhandle, int iterations);

/* ?POTRS: B := A^-1 B for the n x nrhs matrix B, from the Cholesky factor that
 * cu?potrf left in A (same uplo).  LAPACK DPOTRS semantics; the reference library
 * has no ?potrs (its SPD path stops at lapack/dpotrf.c:172 and dpotri.c:25).
 * info = -k when argument k is invalid (XERBLA is called), 0 otherwise. */
CUresult cuDpotrs(CULAPACKhandle, CBlasUplo, size_t, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, long *);
CUresult cuSpotrs(CULAPACKhandle, CBlasUplo, size_t, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, long *);

/* Mixed-precision SPD solve (LAPACK DSPOSV contract; no counterpart in the
 * reference library).  The factor is computed on S A S + shift I, S = diag(A)^-1/2,
 * in FP32 storage: FP64 diagonal blocks, FP32 panel solves, and trailing updates on
 * the tensor cores with BF16 or TF32 operands and FP32 accumulation.  The solve is
 * FP64 preconditioned conjugate gradients on A x = b (FP64 residuals from the
 * caller's A) until every normwise backward error
 *   |b - A x|_inf / (|A|_inf |x|_inf + |b|_inf) <= tol.
 *   cuDcholMixedCreate  scale, factor; keeps the pointer A (read by every solve, so
 *                       leave it unchanged while the plan lives).  shift < 0 picks
 *                       the shift automatically (u/16, u/2, 4u, 32u with u the
 *                       operand unit roundoff 2^-8 or 2^-11, until the factor
 *                       succeeds).
 *                       *info > 0: A has a non-positive diagonal entry at that row,
 *                       or the low-precision factor broke down at that column.
 *   cuDcholMixedSolve   X := A^-1 B (n x nrhs, FP64), tol <= 0 -> sqrt(n) eps,
 *                       maxit <= 0 -> 100 iterations per group of 16 columns;
 *                       *iter = iterations of the slowest group, negative if some
 *                       group did not reach tol; *berr = largest backward error.
 *   cuDposvMixed        one call: create + solve; if the factor breaks down
 *                       (*iter = -3) or the refinement does not converge
 *                       (*iter = -31), A is overwritten by cuDpotrf and X comes
 *                       from cuDpotrf + cuDpotrs (*info as cuDpotrf). */
typedef struct __cucholmixed_st * CUcholMixed;
#define CUCHOL_MIXED_BF16 1
#define CUCHOL_MIXED_TF32 2
CUresult cuDcholMixedCreate(CUcholMixed *, CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, int, double,
                            long *);
CUresult cuDcholMixedSolve(CUcholMixed, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t, double, int, int *,
                           double *);
/* Scale and factor again from the current values of the plan's A (same pointer and
 * order), reusing the plan's buffers; *info as cuDcholMixedCreate. */
CUresult cuDcholMixedRefactor(CUcholMixed, long *);
/* The FP32 factor W (lower, leading dimension *ldw) of S A S + shift I, the FP64
 * scaling vector s, |A|_inf and the shift used (for checking the factor). */
CUresult cuCholMixedGetFactor(CUcholMixed, CUdeviceptr *, size_t *, CUdeviceptr *, double *, double *);
CUresult cuCholMixedDestroy(CUcholMixed);
CUresult cuDposvMixed(CULAPACKhandle, CBlasUplo, size_t, size_t, CUdeviceptr, size_t, CUdeviceptr, size_t,
                      CUdeviceptr, size_t, int, int *, double *, long *);
/* The mixed factor's trailing-update kernel on its own (tcgen05 tensor cores):
 *   C(i, j) += alpha * sum_l Q(i, l) Q(j, l)   for i >= j (lower triangle of C only)
 * with Q an n x k matrix stored k-major (row i at Q + i*ldq elements) in BF16
 * (CUCHOL_MIXED_BF16) or in FP32 words read as TF32 (CUCHOL_MIXED_TF32), C FP32
 * column-major, FP32 accumulation; queued on `stream`.  Q and C 16-byte aligned,
 * ldq * element size and ldc * 4 multiples of 16 bytes (else XERBLA with the position
 * and CUDA_ERROR_INVALID_VALUE). */
CUresult cuSsyrkLowp(CULAPACKhandle, int, size_t, size_t, float, CUdeviceptr, size_t, CUdeviceptr, size_t,
                     CUstream);

/* FP64 Cholesky factor (cuDpotrf contract: in place, info of the first failing
 * leading minor) whose trailing updates run as an Ozaki-sliced emulation on the INT8
 * tensor cores: every panel row is scaled by a power of two and cut into `slices`
 * signed 8-bit slices (4..8; 0 = 8 below n = 8192, 7 from there on), the slice
 * products are exact INT32 sums, and only the final FP64 combination rounds (7 or 8
 * slices: FP64-level backward error).  No counterpart in the reference library. */
CUresult cuDpotrfOzaki(CULAPACKhandle, CBlasUplo, size_t, CUdeviceptr, size_t, int, long *);

/* Random Hermitian positive definite n x n matrix with condition number c, on the
 * device, from the generator's stream (the reference's test generator ?latmc,
 * test/lapack/util/dlatmc.c:11-70, zlatmc.c): D = diag(1, c, d_2 .. d_{n-1}) with d_j
 * uniform in [1, c], u uniform in [0,1] (complex: both parts), and
 * A = H D H^H for the Householder reflection H = I - 2 u u^H / u^H u, so the
 * eigenvalues of A are exactly D's.  Draws, in order, with the generator's [0,1]
 * conversion: d_2 .. d_{n-1}, then u (complex: real and imaginary part of each
 * element in turn).  The full matrix is written (exactly Hermitian); the padding rows
 * are not touched.  Queued on `stream`.  n < 2, c < 1 or lda < n: XERBLA with the
 * position (2, 3, 5) and CUDA_ERROR_INVALID_VALUE. */
CUresult cuSlatmc(CUrng32, size_t, float, CUdeviceptr, size_t, CUstream);
CUresult cuDlatmc(CUrng64, size_t, double, CUdeviceptr, size_t, CUstream);
CUresult cuClatmc(CUrng32, size_t, float, CUdeviceptr, size_t, CUstream);
CUresult cuZlatmc(CUrng64, size_t, double, CUdeviceptr, size_t, CUstream);

/* Counters of a host-memory handle since its creation (for measurement): kernels
 * launched, and bytes copied host -> device and device -> host.  Any pointer may be
 * NULL. */
CUresult cuMultiGPULAPACKGetStats(CUmultiGPULAPACKhandle, unsigned long long *, unsigned long long *,
                                  unsigned long long *);
#ifdef __cplusplus
}
#endif

#endif
