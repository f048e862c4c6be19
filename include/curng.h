/*
 * cucholesky-b200: the GPU pseudo-random number generator API of the reference
 * (include/rng.h:238-413), used to generate inputs on the device.
 *
 * Prototypes are those of the reference.  The generator algorithm is not: the
 * reference ships MTGP (Mersenne Twister for Graphics Processors, parameter set
 * 11213) whose state update is a sequential recurrence split over one block per
 * generator; this library provides Philox4x32-10 (Salmon, Moraes, Dror and Shaw,
 * SC 2011), a counter-based generator whose every 128-bit output block is an
 * independent function of (key, counter), so a fill of any length spreads over
 * the whole GPU and a seed reproduces the same stream at any thread count.  The
 * MTGP types (mtgp32_11213_t, mtgp64_11213_t) are not provided.
 *
 * Stream: word i of a generator seeded with key (k0, k1) is word i mod 4 of
 * Philox4x32-10(counter = (b mod 2^32, b div 2^32, 0, 0), key), b = i div 4.
 * cuRng32 values are words; cuRng64 values are two consecutive words (the first is
 * the low half).  Every fill starts at a fresh 128-bit block after the previous
 * one, so consecutive calls continue the stream.  Float conversions (exact):
 *   32-bit: [0,1) (w >> 8) 2^-24;  (0,1] ((w >> 8) + 1) 2^-24;
 *           (0,1) ((w >> 9) + 1/2) 2^-23;  [0,1] (w >> 8) / (2^24 - 1)
 *   64-bit: [0,1) (x >> 11) 2^-53; (0,1] ((x >> 11) + 1) 2^-53;
 *           (0,1) ((x >> 12) + 1/2) 2^-52; [0,1] (x >> 11) / (2^53 - 1)
 * Fills are queued on the legacy default stream and return without waiting.
 */
#ifndef CUCHOLESKY_CURNG_H
#define CUCHOLESKY_CURNG_H

#include <stddef.h>
#include <stdint.h>
#include <cuda.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct __curng32_type_st * CUrng32_t;   /* rng.h:241 */
typedef struct __curng32_st * CUrng32;          /* rng.h:246 */
typedef struct __curng64_type_st * CUrng64_t;   /* rng.h:330 */
typedef struct __curng64_st * CUrng64;          /* rng.h:335 */

/* Philox4x32-10 for cuRng32Create / cuRng64Create. */
extern const CUrng32_t philox32_t;
extern const CUrng64_t philox64_t;

/* Create (seed 0), destroy, seed (key = the seed; the stream restarts at word 0)
 * (reference include/rng.h:257-272, 346-361). */
CUresult cuRng32Create(CUrng32 *, const CUrng32_t);
CUresult cuRng32Destroy(CUrng32);
CUresult cuRng32Set(const CUrng32, uint32_t);
/* n 32-bit words, or floats in (0,1), (0,1], [0,1), [0,1] (rng.h:281-321). */
CUresult cuRng32Get(const CUrng32, CUdeviceptr, size_t);
CUresult cuRng32GetOpenOpen(const CUrng32, CUdeviceptr, size_t);
CUresult cuRng32GetOpenClose(const CUrng32, CUdeviceptr, size_t);
CUresult cuRng32GetCloseOpen(const CUrng32, CUdeviceptr, size_t);
CUresult cuRng32GetCloseClose(const CUrng32, CUdeviceptr, size_t);

CUresult cuRng64Create(CUrng64 *, const CUrng64_t);
CUresult cuRng64Destroy(CUrng64);
CUresult cuRng64Set(const CUrng64, uint64_t);
/* n 64-bit integers, or doubles in (0,1), (0,1], [0,1), [0,1] (rng.h:370-410). */
CUresult cuRng64Get(const CUrng64, CUdeviceptr, size_t);
CUresult cuRng64GetOpenOpen(const CUrng64, CUdeviceptr, size_t);
CUresult cuRng64GetOpenClose(const CUrng64, CUdeviceptr, size_t);
CUresult cuRng64GetCloseOpen(const CUrng64, CUdeviceptr, size_t);
CUresult cuRng64GetCloseClose(const CUrng64, CUdeviceptr, size_t);

#ifdef __cplusplus
}
#endif

#endif
