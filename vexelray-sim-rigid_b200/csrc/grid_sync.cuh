// A grid-wide barrier for a cooperative (all blocks co-resident) launch, with a bounded wait.
//
// Arrival is an atomic add on a counter; the last block to arrive resets it and bumps a generation word the
// others poll. Every wait gives up after a time limit (the device's global nanosecond timer): the waiter then
// raises the abort word and the status word, and every block leaves at its next barrier, so a barrier that can
// never complete ends the kernel with an error the host reads, not a hung GPU.
#pragma once
#include <cstdint>

namespace vxr {

enum : int { ST_OK = 0, ST_CAPACITY = 2, ST_ROUNDS = 3, ST_NONFINITE = 4, ST_TIMEOUT = 5 };

struct GridBarrier {
    unsigned int* count;       // arrivals this generation
    unsigned int* generation;  // bumped once per completed barrier
    int* abort;                // nonzero: every block leaves
    int* status;               // the step's status word
    unsigned long long limit_ns;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Returns false when the kernel must stop (a wait ran out here or elsewhere).
__device__ __forceinline__ bool grid_sync(const GridBarrier& b) {
    __syncthreads();
    __shared__ int leave;
    if (threadIdx.x == 0) {
        leave = 0;
        volatile unsigned int* gen = b.generation;
        const unsigned int g = *gen;
        __threadfence();
        const unsigned int arrived = atomicAdd(b.count, 1u);
        if (arrived == gridDim.x - 1) {
            *b.count = 0u;
            __threadfence();
            atomicAdd(b.generation, 1u);
        } else {
            const unsigned long long start = global_ns();
            unsigned int spins = 0;
            while (*gen == g) {
                if (*(volatile int*)b.abort) break;
                if ((++spins & 63u) == 0u && global_ns() - start > b.limit_ns) {
                    atomicExch(b.abort, 1);
                    atomicCAS(b.status, ST_OK, ST_TIMEOUT);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (*(volatile int*)b.abort) leave = 1;
    }
    __syncthreads();
    return leave == 0;
}

}  // namespace vxr
