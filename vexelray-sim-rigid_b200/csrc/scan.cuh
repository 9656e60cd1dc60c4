// Device-wide exclusive prefix sum of int32 counts, in three launches: per-block sums, a scan of the block sums in
// one block, and the per-block scan with its offset. out[n] receives the total. Used for the cell starts of the
// counting sort and for every compaction of the step (candidate pairs, touching pairs, incidence lists, rounds).
#pragma once
#include <cuda_runtime.h>

namespace vxr {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_sums, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    const int before = warp > 0 ? warp_sums[warp - 1] : 0;
    total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void k_scan_tiles(const int* __restrict__ in, int n, int* __restrict__ tile_sums) {
    __shared__ int ws[32];
    const long base = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_ITEMS;
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
        if (base + i < n) s += in[base + i];
    int total;
    block_exclusive_scan(s, ws, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(int* tile_sums, int tiles, int* __restrict__ out, int n) {
    __shared__ int ws[32];
    int carry = 0;
    for (int start = 0; start < tiles; start += SCAN_THREADS) {
        const int i = start + threadIdx.x;
        const int v = i < tiles ? tile_sums[i] : 0;
        int total;
        const int ex = block_exclusive_scan(v, ws, total);
        if (i < tiles) tile_sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) out[n] = carry;
}

__global__ void k_scan_apply(const int* __restrict__ in, int n, const int* __restrict__ tile_sums,
                             int* __restrict__ out) {
    __shared__ int ws[32];
    const long base = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = base + i < n ? in[base + i] : 0;
        s += v[i];
    }
    int total;
    int run = block_exclusive_scan(s, ws, total) + tile_sums[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

// Exclusive scan of in[0..n) into out[0..n], out[n] = total. tile_sums holds ceil(n / SCAN_TILE) ints.
inline void exclusive_scan(const int* in, int* out, int n, int* tile_sums, cudaStream_t st) {
    const int tiles = n > 0 ? (n + SCAN_TILE - 1) / SCAN_TILE : 1;
    if (n > 0) k_scan_tiles<<<tiles, SCAN_THREADS, 0, st>>>(in, n, tile_sums);
    else cudaMemsetAsync(tile_sums, 0, sizeof(int), st);
    k_scan_sums<<<1, SCAN_THREADS, 0, st>>>(tile_sums, n > 0 ? tiles : 0, out, n);
    if (n > 0) k_scan_apply<<<tiles, SCAN_THREADS, 0, st>>>(in, n, tile_sums, out);
}

inline int scan_tiles_for(int n) { return n > 0 ? (n + SCAN_TILE - 1) / SCAN_TILE : 1; }

}  // namespace vxr
