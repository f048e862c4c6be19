/*
 * cucholesky-b200: the device-list object of the reference's host-memory LAPACK
 * routines (reference include/cumultigpu.h).
 *
 * A CUmultiGPU names the GPUs that a CUmultiGPULAPACKhandle (include/lapack.h)
 * may use.  The reference backed it with one worker thread and CUDA context per
 * device and a task queue (multigpu/multigpu.c); this library keeps only the
 * device list: its host-memory routines stage the matrix into one GPU's memory
 * and run the single-GPU path there, because one factorization fits a B200's
 * 180 GB and its panel chain does not shard.  The reference's task API
 * (CUtask, cuTaskCreate/Destroy/Execute, cuMultiGPURunTask) is not provided.
 *
 * Prototypes are those of the reference (line numbers cited per entry).
 */
#ifndef CUCHOLESKY_CUMULTIGPU_H
#define CUCHOLESKY_CUMULTIGPU_H

#include <stddef.h>
#include <cuda.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct __cumultigpu_st * CUmultiGPU;

/* Device list of n >= 1 CUDA devices (ordinals as returned by cuDeviceGet;
 * repeats allowed).  CUDA_ERROR_INVALID_VALUE for a NULL pointer or n < 1,
 * CUDA_ERROR_INVALID_DEVICE for an ordinal that does not exist
 * (reference include/cumultigpu.h:61, multigpu/multigpu.c:437). */
CUresult cuMultiGPUCreate(CUmultiGPU *, CUdevice *, int);

/* Frees the list; waits for nothing (reference include/cumultigpu.h:69). */
CUresult cuMultiGPUDestroy(CUmultiGPU);

/* Number of devices in the list, 0 for NULL (reference include/cumultigpu.h:77). */
int cuMultiGPUGetContextCount(CUmultiGPU);

/* Waits for all work on every listed device (reference include/cumultigpu.h:97). */
CUresult cuMultiGPUSynchronize(CUmultiGPU);

#ifdef __cplusplus
}
#endif

#endif
