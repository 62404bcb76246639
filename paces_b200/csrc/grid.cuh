// Bounded grid-wide barrier of the persistent cooperative kernels (the Taylor series).
#pragma once

#include "common.cuh"

namespace paces {

// All blocks are co-resident (cooperative launch).  bar[0] counts arrivals, bar[1] is the
// generation; a wait longer than `limit_ns` raises PACES_ERR_TIMEOUT on `status` (if given)
// and returns false instead of spinning on.  `skip` (a test hook) makes this block give up
// without arriving: it raises the timeout itself, and every other block's wait runs out.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned nblocks, unsigned& gen, int* status,
                                             uint64_t limit_ns = kWaitLimitNs, bool skip = false) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0 && skip) {
        raise_status(status, PACES_ERR_TIMEOUT);
        s_ok = 0;
    } else if (threadIdx.x == 0) {
        s_ok = 1;
        __threadfence();
        const unsigned arrived = atomicAdd(&bar[0], 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            const uint64_t t0 = global_ns();
            while (atomicAdd(&bar[1], 0u) == gen) {
                if (global_ns() - t0 > limit_ns) {
                    raise_status(status, PACES_ERR_TIMEOUT);
                    s_ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        ++gen;
        __threadfence();
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace paces
