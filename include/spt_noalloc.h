/*
 * spt_noalloc.h -- an entry point of the B200 backend that allocates nothing during the call.
 *
 * No reference counterpart: the reference's AccelStructure::intersect (acceleration/accel_structure.h:29-30)
 * works on one ray at a time in host memory and has no device scratch.  This is spt_intersect (spt.h)
 * for callers that cannot let a call allocate or free device memory: cudaFree waits for all work on the
 * device, which a caller sharing the device with other busy streams cannot afford, and cudaMalloc can
 * fail for a caller that has already reserved the device's memory for itself.
 *
 * Same results and semantics as spt_intersect, with these limits:
 *   - at most 65536 rays per call (the size of the static device buffer that holds rays, hits and
 *     counts, 3.5 MiB per device); larger batches return SPT_ERR_INVALID_ARGUMENT and must be split;
 *   - the static buffer is shared by every context of the process on that device: calls that overlap
 *     in time on one device (from two threads, or on two contexts' streams) race on it, so the caller
 *     serialises them;
 *   - the first call with a context looks the buffer up (cudaGetSymbolAddress, which may load the
 *     library's module) and keeps its address in the context: make that call before any stream
 *     capture starts on the device.
 */
#ifndef SPT_NOALLOC_H
#define SPT_NOALLOC_H

#include "spt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* rays: n x 8 floats (host); hits: n records (host); tests / nhits (host, may be NULL): the reference's
 * per-ray num_intersection_tests / num_intersections.  Returns after the results are in host memory. */
spt_status spt_intersect_noalloc(spt_context* ctx, const spt_scene* scene, const float* rays, uint64_t n,
                                 spt_hit* hits, uint32_t* tests, uint32_t* nhits);

#ifdef __cplusplus
}
#endif

#endif /* SPT_NOALLOC_H */
