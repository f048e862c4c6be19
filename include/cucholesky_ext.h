/*
 * Extensions of libcucholesky.so beyond the reference API.  Same conventions as
 * include/lapack.h (handle first, CUresult return, host `long *info`).  None of
 * these has a counterpart in the reference library.
 */
#ifndef CUCHOLESKY_EXT_H
#define CUCHOLESKY_EXT_H

#include "lapack.h"

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

#ifdef __cplusplus
}
#endif

#endif
