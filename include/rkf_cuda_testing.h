/*
 * rkf_cuda_testing.h — failure injection for tests of the engine's error
 * paths.  No counterpart in the reference.  The failure is made on the host:
 * no GPU fault is ever provoked.
 */
#ifndef RKF_CUDA_TESTING_H
#define RKF_CUDA_TESTING_H

#include "rkf_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* After n more successful device allocations by any context, the next one
 * reports out-of-memory (RKF_OOM) without calling cudaMalloc; n < 0 turns
 * the injection off.  Process-wide. */
RKF_API void rkf_testing_fail_allocation_after(long long n);

/* Copy the empty-space distance field (one byte per top-grid cell, indexed
 * like the top grid of rkf_index_export: 0 for a block that is not EMPTY,
 * else the Chebyshev distance in blocks to the nearest such block of the
 * same object, capped at 64) into out (may be NULL); *n receives the cell
 * count. */
RKF_API rkf_status rkf_testing_export_empty_dist(rkf_ctx* ctx, uint8_t* out, uint64_t* n);

/* Number of bands rkf_march uses for a view with host outputs (1 = one
 * launch, then the copies; at most 8), whatever the view's size and whether
 * or not its planes are page-locked; bands < 0 restores the choice by view
 * size (page-locked planes only).  Process-wide. */
RKF_API void rkf_testing_set_host_bands(int bands);

/* The tiled strategy's coarse field for the context's current objects (built
 * if needed): its origin, dims and, when tex is not NULL, its dims[0] x
 * dims[1] x dims[2] binary16 texels (x + y*dx + z*dx*dy); *n receives the
 * texel count. */
RKF_API rkf_status rkf_testing_export_coarse(rkf_ctx* ctx, float origin[3], uint32_t dims[3], uint16_t* tex,
                                             uint64_t* n);

/* Kernel variant of the context's last march launch through rkf_march,
 * rkf_march_rays or rkf_march_batch: 0 several objects, 1 one object, 2 one
 * object on the empty-space path, 3 the same under the tiled strategy, 4
 * several objects on the multi-object empty-space path, 5 the same under the
 * tiled strategy; -1 before the first. */
RKF_API int rkf_testing_last_variant(rkf_ctx* ctx);

/* The multi-object empty-space path's ball of an analytic object, for EMPTY
 * values up to empty_hi: out = {centre x, y, z, a, b}, radius a + b*P where P
 * bounds |o| + |d| |tmax| of a ray.  Every value the object takes outside the
 * ball exceeds empty_hi.  Host only (no device is touched).  1 when the
 * object has a ball; 0 for a plane, a singular or ill-conditioned
 * transform, a non-positive scale or non-finite parameters. */
RKF_API int rkf_testing_far_ball(const rkf_gpu_object* obj, float empty_hi, float out[5]);

/* The multi-object empty-space path's half-space of an analytic plane, for
 * EMPTY values up to empty_hi: out = {G x, y, z, H, a, b}; wherever a
 * position w with |w|_1 <= P has G.w + H > a + b*P, the plane's value
 * exceeds empty_hi.  Host only.  1 for a plane with a finite transform and
 * a non-zero normal, else 0. */
RKF_API int rkf_testing_far_plane(const rkf_gpu_object* obj, float empty_hi, float out[6]);

/* Brick-pool and index-leaf bookkeeping: out = {pool capacity, live bricks
 * (pool_bricks_used), free slots, leaf blocks allocated, free leaf blocks}.
 * Slots neither live nor free are held for work of older epochs.  Read it
 * while no edit runs (a serving session between requests, or no session). */
RKF_API rkf_status rkf_testing_pool_state(rkf_ctx* ctx, uint32_t out[5]);

/* Launch accounting.  enable = 1 starts timing the context's persistent
 * march launches (the kernel of rkf_march, rkf_march_async,
 * rkf_march_rays, rkf_march_batch and their variants) with a pair of CUDA
 * events on each launch's stream around the kernel alone, discarding the
 * launches timed before; 0 stops it.  At most 4096 launches are timed.
 * RKF_BUSY while a serving session runs. */
RKF_API rkf_status rkf_testing_march_timing(rkf_ctx* ctx, uint32_t enable);

/* *launches (may be NULL): kernels the context has launched since it was
 * created, on any stream (march, tile order, tiled-strategy preparation,
 * voxelization, edits, imports, queries).  *n_timed (may be NULL): launches
 * timed since timing was switched on; march_ms[i] receives the device time
 * of the i-th of them, for i < min(cap, *n_timed), waiting for each to
 * finish. */
RKF_API rkf_status rkf_testing_launch_stats(rkf_ctx* ctx, uint64_t* launches, float* march_ms, uint32_t cap,
                                            uint32_t* n_timed);

#ifdef __cplusplus
}
#endif
#endif /* RKF_CUDA_TESTING_H */
