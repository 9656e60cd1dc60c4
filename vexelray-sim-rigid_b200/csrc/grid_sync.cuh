// A grid-wide barrier for a cooperative (all blocks co-resident) launch, with a bounded wait.
//
// Arrival is one release-ordered add per block on a counter that only grows during the kernel (zeroed before the
// launch), and the wait an acquire load of it: barrier number e is passed once the counter reaches (e + 1) x blocks, so no block resets anything
// and no second word is needed. Every wait gives up after a time limit (the device's global nanosecond timer):
// the waiter then raises the abort word and the status word, and every block leaves at its next barrier, so a
// barrier that can never complete ends the kernel with an error the host reads, not a hung GPU.
#pragma once
#include <cstdint>

namespace vxr {

enum : int { ST_OK = 0, ST_CAPACITY = 2, ST_ROUNDS = 3, ST_NONFINITE = 4, ST_TIMEOUT = 5 };

struct GridBarrier {
    unsigned int* count;       // arrivals since the launch
    unsigned int* generation;  // unused by this barrier; kept zero
    int* abort;                // nonzero: every block leaves
    int* status;               // the step's status word
    unsigned long long limit_ns;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int load_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Returns false when the kernel must stop (a wait ran out here or elsewhere). `epoch` counts this block's
// barriers since the launch; every block passes the same barriers in the same order.
__device__ __forceinline__ bool grid_sync(const GridBarrier& b, unsigned int& epoch) {
    __syncthreads();
    __shared__ int leave;
    if (threadIdx.x == 0) {
        leave = 0;
        const unsigned int target = (epoch + 1) * gridDim.x;
        // Arrival as a release at GPU scope: the block's writes (ordered before it by the block barrier) are
        // visible to every block whose acquire load then sees the count. No separate full fence is needed.
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(b.count), "r"(1u) : "memory");
        if (load_acquire(b.count) < target) {
            const unsigned long long start = global_ns();
            unsigned int spins = 0;
            while (load_acquire(b.count) < target) {
                if (*(volatile int*)b.abort) break;
                if (((++spins & 255u) == 0u || spins == 1u) && global_ns() - start > b.limit_ns) {
                    atomicExch(b.abort, 1);
                    atomicCAS(b.status, ST_OK, ST_TIMEOUT);
                    break;
                }
            }
        }
        if (*(volatile int*)b.abort) leave = 1;
    }
    epoch++;
    __syncthreads();
    return leave == 0;
}

}  // namespace vxr
