// gg_grid.cuh -- helpers of the cooperative (persistent) kernels: the global
// timer and a bounded grid barrier.
//
// The barrier is the persistent kernels' only wait.  It is bounded by a
// %globaltimer deadline; a CTA that gives up sets DEV_ERR_TIMEOUT in *err and
// returns false, and every CTA leaves at its next barrier, so the host gets
// GG_ERR_TIMEOUT and the context stays usable.  Co-residency of all CTAs is
// guaranteed by the cooperative launch, so in normal operation the deadline
// is never reached.
#pragma once
#include "gg_internal.cuh"

namespace gg {
namespace grid {

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct Barrier {
    unsigned int count;
    unsigned int gen;
    unsigned int err;
};

__device__ __forceinline__ bool sync(Barrier *b, unsigned long long timeout_ns) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        volatile unsigned int *genp = &b->gen;
        const unsigned int gen = *genp;
        if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            const unsigned long long t0 = globaltimer();
            while (*genp == gen) {
                if (globaltimer() - t0 > timeout_ns) {
                    atomicOr(&b->err, DEV_ERR_TIMEOUT);
                    break;
                }
                if (*(volatile unsigned int *)&b->err) break;
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile unsigned int *)&b->err == 0;
}

}  // namespace grid
}  // namespace gg
