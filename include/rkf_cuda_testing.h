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

#ifdef __cplusplus
}
#endif
#endif /* RKF_CUDA_TESTING_H */
