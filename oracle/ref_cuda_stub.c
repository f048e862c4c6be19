/* Host-only stand-ins for the CUDA driver entry points that the reference's GPU
 * halves reference from the same translation units as its CPU routines
 * (lapack/*.c, blas/*.c, multigpu/multigpu.c).  The CPU routines never call them;
 * if anything does, it gets 801 (CUDA_ERROR_NOT_SUPPORTED).  cuda.h is not
 * included on purpose: only the link-time names matter here.  Test
 * infrastructure only. */
#define STUB(name) int name(void) { return 801; }
STUB(cuCtxCreate_v2) STUB(cuCtxDestroy_v2) STUB(cuCtxGetCurrent) STUB(cuCtxPopCurrent_v2)
STUB(cuCtxPushCurrent_v2) STUB(cuCtxSynchronize) STUB(cuDeviceGet) STUB(cuGetErrorString)
STUB(cuLaunchKernel) STUB(cuMemAllocHost_v2) STUB(cuMemAllocPitch_v2) STUB(cuMemAlloc_v2)
STUB(cuMemFreeHost) STUB(cuMemFree_v2) STUB(cuMemcpy2DAsync_v2) STUB(cuMemcpyDtoHAsync_v2)
STUB(cuMemcpyHtoDAsync_v2) STUB(cuModuleGetFunction) STUB(cuModuleLoadData) STUB(cuModuleUnload)
STUB(cuStreamCreate) STUB(cuStreamDestroy_v2) STUB(cuStreamSynchronize)
