// wf_gridbar.cuh - bounded grid-wide barrier of the persistent (cooperative)
// loop kernels (wf_sweeps.cu, wf_nonuniform.cu).
#pragma once
#include <cuda_runtime.h>

#include "wf_sweeps.cuh"

namespace wf {

__device__ __forceinline__ unsigned long long gridbar_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier for `expected` arriving blocks.  Returns false (on every
// thread of the block) when the barrier's error word is or becomes set, or
// when this block waited longer than timeout_ns.
__device__ __forceinline__ bool grid_barrier(GridBar* bar, unsigned expected, unsigned long long timeout_ns) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
        volatile GridBar* vb = bar;
        int good = vb->err == 0;
        if (good) {
            const unsigned gen = vb->gen;
            __threadfence();
            const unsigned arrived = atomicAdd(&bar->count, 1u) + 1u;
            if (arrived == expected) {
                bar->count = 0;
                __threadfence();
                atomicAdd(&bar->gen, 1u);
            } else {
                const unsigned long long t0 = gridbar_ns();
                while (vb->gen == gen) {
                    if (vb->err != 0) {
                        good = 0;
                        break;
                    }
                    if (gridbar_ns() - t0 > timeout_ns) {
                        atomicExch(&bar->err, 1);
                        good = 0;
                        break;
                    }
                    __nanosleep(64);
                }
            }
            __threadfence();
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace wf
