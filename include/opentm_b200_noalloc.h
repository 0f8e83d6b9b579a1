/*
 * opentm_b200_noalloc.h -- entry point of the B200 library that allocates no device memory.
 *
 * Some callers cannot allocate GPU memory while they run: a framework whose caching allocator
 * has already reserved the device's memory for itself, a latency-critical loop where a
 * cudaMalloc/cudaFree (which can synchronize the whole device and take milliseconds) is not
 * allowed, or a host whose policy forbids run-time device allocations. For them this header
 * offers the OC sensitivity filter with its temporary copy in a fixed, statically sized
 * device array instead of memory allocated per call.
 */
#ifndef OPENTM_B200_NOALLOC_H
#define OPENTM_B200_NOALLOC_H

#include "opentm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Largest cell (voxels) the allocation-free filter accepts: 2^21 = 128^3. The library holds
 * a static device array of this many floats (8 MiB) on every GPU that loads it, until the
 * process exits. */
#define OTM_NOALLOC_MAX_CELLS (1 << 21)

/* No counterpart in the reference: the same filter as otm_oc_filter_sens (the reference's
 * OCOptimizer::filterSens allocates and frees a temporary buffer on every call), but the
 * temporary lives in the library's static device array, so the call allocates nothing.
 * Returns OTM_ERR_UNSUPPORTED for a cell of more than OTM_NOALLOC_MAX_CELLS voxels.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture. With lazy module loading (the CUDA default) that
 * first call is also when the library's device code is loaded and the 8 MiB array is reserved on
 * the device, so make it (a warm-up call on a small cell will do) before the caller's own
 * allocator takes the device's memory. The address is kept per device for the life of the
 * process: do not use this entry point across a cudaDeviceReset of that device. All calls share
 * the one array: calls whose GPU
 * work overlaps (several streams or host threads at once) race on it, so order them on one
 * stream. The array keeps the last call's contents; nothing in it needs to start at zero,
 * because every element a call reads was written earlier in the same call. */
OTM_API otm_status otm_oc_filter_sens_noalloc(float* sens, const float* rho, size_t pitchT, const int reso[3],
                                              float radius, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OPENTM_B200_NOALLOC_H */
