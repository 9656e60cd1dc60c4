// The learned warm start's network on the 5th-generation tensor cores: a 16 -> 64 -> 64 -> 2 multilayer perceptron
// with SiLU activations, BF16 weights and activations, FP32 accumulation in tensor memory. No reference
// counterpart: the reference warm-starts a contact with last step's impulses (core/box/BoxPairs.java:191-267,
// core/sphere/Spheres.java:448-481); this network predicts a contact's starting normal and friction impulse from
// local features instead.
//
// Every product is one tcgen05.mma (kind::f16, BF16 x BF16 -> F32, M = 128) issued by one thread, operands in shared
// memory in the no-swizzle K-major layout (8-row x 16-byte core matrices; LBO steps along K, SBO along M or N), the
// accumulator in tensor memory, read back by a warpgroup with tcgen05.ld (row i of the tile is lane i). A tile is 128
// contacts, one thread each.
//   forward:  Z1 = X W1, Z2 = H1 W2, Y = H2 W3                       (K = 16, 64, 64; N = 64, 64, 16)
//   backward: dH2 = D3 W3^T, dH1 = D2 W2^T                            (K = 16, 64;    N = 64, 64)
//             [dW2 | . ; . | dW1 ; db2 | db1] = [H1^T ; X^T ; 1] [D2 | D1]     (one M = 128, N = 128, K = 128 product)
//             [dW3 ; db3] = [H2^T ; 1] D3                                        (M = 128, N = 16, K = 128)
// Every wait on an mbarrier is bounded: past the limit the kernel records an error, waits (bounded again) for its
// own products in flight, frees its tensor memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "vxr.h"

namespace vxr {
namespace mlp {

constexpr int IN = 16, HID = 64, OUT = 2, TILE = 128, THREADS = 128;
// the FP32 master parameters, in this order: w1 [16][64], b1 [64], w2 [64][64], b2 [64], w3 [64][2], b3 [2]
constexpr int O_W1 = 0, O_B1 = O_W1 + IN * HID, O_W2 = O_B1 + HID, O_B2 = O_W2 + HID * HID, O_W3 = O_B2 + HID,
              O_B3 = O_W3 + HID * OUT, N_PARAMS = O_B3 + OUT;
static_assert(N_PARAMS == VXR_MLP_PARAMS, "parameter count");
// Tensor-memory columns a block takes: the forward's three products fit in 128 (four blocks an SM fill the 512
// columns exactly, so an allocation never waits); the training kernel (one block an SM) takes 256.
constexpr uint32_t FWD_COLS = 128, TRAIN_COLS = 256;
constexpr unsigned long long WAIT_NS = 2000000000ull;  // 2 s: far above any product's honest wait

// Byte offset of element (r, k) of a K-major operand with `rows` rows: core matrices of 8 rows x 8 BF16, all the
// row groups of K-chunk 0, then of K-chunk 1, ... So SBO (next 8 rows) = 128 B and LBO (next 8 of K) = rows x 16 B.
__host__ __device__ constexpr uint32_t kmaj(int r, int k, int rows) {
    return (uint32_t)((((k >> 3) * (rows >> 3) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared memory matrix descriptor: start, LBO, SBO (16-byte units), version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t start, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// The operand descriptor of K-step s (16 of K) of a `rows`-row K-major operand at `base`.
__device__ __forceinline__ uint64_t operand(uint32_t base, int rows, int s) {
    return sdesc(base + (uint32_t)(2 * s * rows * 16), (uint32_t)(rows * 16), 128u);
}

// Instruction descriptor: F32 accumulator, BF16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d), "l"(a), "l"(b), "r"(id), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the mbarrier's phase `parity` to complete; gives up after WAIT_NS of the device's clock.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    const unsigned long long start = now_ns();
    for (unsigned i = 1;; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 63u) == 0u && now_ns() - start > WAIT_NS) return false;
    }
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld_x16(uint32_t taddr, uint32_t* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld_x64(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, "
        "%36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, "
        "%57, %58, %59, %60, %61, %62, %63}, [%64];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
}

__device__ __forceinline__ void put(uint8_t* tile, int r, int k, int rows, float v) {
    *(__nv_bfloat16*)(tile + kmaj(r, k, rows)) = __float2bfloat16_rn(v);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// The network as the kernels read it: BF16 operand views of the weights (each in the K-major orientation its
// product needs) and the FP32 biases and feature normalisation.
struct Net {
    const __nv_bfloat16* w1t;  // [64][16]  W1^T      (forward B, layer 1)
    const __nv_bfloat16* w2t;  // [64][64]  W2^T      (forward B, layer 2)
    const __nv_bfloat16* w3t;  // [16][64]  W3^T, rows 2.. zero (forward B, layer 3)
    const __nv_bfloat16* w2n;  // [64][64]  W2        (backward B, dH1)
    const __nv_bfloat16* w3n;  // [64][16]  W3, cols 2.. zero (backward B, dH2)
    const float* master;       // FP32 parameters (biases read from here)
    const float* mean;         // [16]
    const float* inv_std;      // [16]
};

// Shared memory of both kernels (bytes); the forward uses the first part.
constexpr uint32_t S_XA = 0;                  // X      128 x 16
constexpr uint32_t S_W1 = S_XA + 128 * 16 * 2;  // W1^T    64 x 16
constexpr uint32_t S_H1 = S_W1 + 64 * 16 * 2;   // H1     128 x 64
constexpr uint32_t S_W2 = S_H1 + 128 * 64 * 2;  // W2^T    64 x 64
constexpr uint32_t S_H2 = S_W2 + 64 * 64 * 2;   // H2     128 x 64
constexpr uint32_t S_W3 = S_H2 + 128 * 64 * 2;  // W3^T    16 x 64
constexpr uint32_t S_FWD_END = S_W3 + 16 * 64 * 2;
constexpr uint32_t S_D3 = S_FWD_END;            // D3     128 x 16
constexpr uint32_t S_W3N = S_D3 + 128 * 16 * 2; // W3      64 x 16
constexpr uint32_t S_D2 = S_W3N + 64 * 16 * 2;  // D2     128 x 64
constexpr uint32_t S_W2N = S_D2 + 128 * 64 * 2; // W2      64 x 64
constexpr uint32_t S_AG = S_W2N + 64 * 64 * 2;  // [H1^T; X^T; 1]  128 x 128 (K = samples)
constexpr uint32_t S_BG = S_AG + 128 * 128 * 2; // [D2^T; D1^T]    128 x 128
constexpr uint32_t S_A3 = S_BG + 128 * 128 * 2; // [H2^T; 1]       128 x 128
constexpr uint32_t S_B3 = S_A3 + 128 * 128 * 2; // D3^T             16 x 128
constexpr uint32_t S_TRAIN_END = S_B3 + 16 * 128 * 2;
constexpr uint32_t FWD_SMEM = S_FWD_END + 16, TRAIN_SMEM = S_TRAIN_END + 16;

template <int ROWS, int K>
__device__ __forceinline__ void load_view(uint8_t* tile, const __nv_bfloat16* view) {
    for (int i = threadIdx.x; i < ROWS * K; i += THREADS) {
        const int r = i / K, k = i % K;
        *(__nv_bfloat16*)(tile + kmaj(r, k, ROWS)) = view[i];
    }
}

// Tensor memory for the block: warp 0 allocates, every thread reads the address.
__device__ __forceinline__ uint32_t tmem_take(uint32_t* slot, uint32_t cols) {
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)),
                     "r"(cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    return *(volatile uint32_t*)slot;
}

__device__ __forceinline__ void tmem_give(uint32_t tmem, uint32_t cols) {
    fence_before();
    __syncthreads();
    fence_after();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols));
}

__device__ __forceinline__ void bar_init(uint64_t* bar) {
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
}

// What every thread does between writing a product's operands and the one thread issuing it.
__device__ __forceinline__ void operands_ready() {
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
}

// The wait for the products just committed, the same verdict in every thread. On a timeout: record it, wait once
// more (bounded) for the products in flight, and report false so the kernel frees its tensor memory and leaves.
__device__ __forceinline__ bool products_done(uint32_t bar, uint32_t& phase, int* status) {
    bool ok = mbar_wait(bar, phase);
    ok = __syncthreads_and(ok) != 0;
    if (!ok) {
        if (threadIdx.x == 0) atomicExch(status, VXR_ETIMEOUT);
        mbar_wait(bar, phase);
    }
    phase ^= 1u;
    fence_after();
    return ok;
}

__device__ __forceinline__ int row_count(const int* rows_dev, int rows_mult, int rows_host) {
    return rows_dev ? (*(const volatile int*)rows_dev) * rows_mult : rows_host;
}

// Forward over `rows` feature rows (rows_dev: a device count times rows_mult, when the count is only known on the
// device): out[r] = (normal, friction) predicted.
__global__ void __launch_bounds__(THREADS, 1) k_mlp_forward(Net net, const float* __restrict__ feats,
                                                            const int* rows_dev, int rows_mult, int rows_host,
                                                            float* __restrict__ out, int* status) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint64_t* bar = (uint64_t*)(sm + S_FWD_END);
    uint32_t* slot = (uint32_t*)(sm + S_FWD_END + 8);
    const int tid = threadIdx.x, warp = tid >> 5;
    load_view<64, 16>(sm + S_W1, net.w1t);
    load_view<64, 64>(sm + S_W2, net.w2t);
    load_view<16, 64>(sm + S_W3, net.w3t);
    bar_init(bar);
    const uint32_t tmem = tmem_take(slot, FWD_COLS);
    const uint32_t lane = (uint32_t)(warp * 32) << 16;
    const uint32_t b = saddr(bar);
    const float* b1 = net.master + O_B1;
    const float* b2 = net.master + O_B2;
    const float* b3 = net.master + O_B3;
    uint32_t phase = 0;
    const int rows = row_count(rows_dev, rows_mult, rows_host);
    const int tiles = (rows + TILE - 1) / TILE;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int r = t * TILE + tid;
        const bool valid = r < rows;
#pragma unroll
        for (int j = 0; j < IN; j++) {
            const float v = valid ? (feats[(size_t)r * IN + j] - net.mean[j]) * net.inv_std[j] : 0.0f;
            put(sm + S_XA, tid, j, 128, v);
        }
        operands_ready();
        if (tid == 0) {
            mma(tmem, operand(saddr(sm + S_XA), 128, 0), operand(saddr(sm + S_W1), 64, 0), idesc(128, 64), 0);
            commit(b);
        }
        if (!products_done(b, phase, status)) break;
        uint32_t v[64];
        tmem_ld_x64(tmem + lane, v);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < HID; j++) put(sm + S_H1, tid, j, 128, silu(__uint_as_float(v[j]) + b1[j]));
        operands_ready();
        if (tid == 0) {
            for (int s = 0; s < 4; s++)
                mma(tmem + 64, operand(saddr(sm + S_H1), 128, s), operand(saddr(sm + S_W2), 64, s), idesc(128, 64),
                    s > 0);
            commit(b);
        }
        if (!products_done(b, phase, status)) break;
        tmem_ld_x64(tmem + lane + 64, v);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < HID; j++) put(sm + S_H2, tid, j, 128, silu(__uint_as_float(v[j]) + b2[j]));
        operands_ready();
        if (tid == 0) {
            for (int s = 0; s < 4; s++)
                mma(tmem, operand(saddr(sm + S_H2), 128, s), operand(saddr(sm + S_W3), 16, s), idesc(128, 16),
                    s > 0);  // columns 0-15: layer 1's, read already
            commit(b);
        }
        if (!products_done(b, phase, status)) break;
        uint32_t y[16];
        tmem_ld_x16(tmem + lane, y);
        tmem_wait_ld();
        if (valid) {
            out[(size_t)r * OUT] = __uint_as_float(y[0]) + b3[0];
            out[(size_t)r * OUT + 1] = __uint_as_float(y[1]) + b3[1];
        }
        fence_before();
        __syncthreads();
        fence_after();
    }
    tmem_give(tmem, FWD_COLS);
}

// Forward and backward over one batch: every block takes tiles of the batch's rows (rows index[r] of the data, or r
// itself), and adds its tiles' gradients of the loss sum |y - t|^2 / batch to grads (FP32, the master layout) and
// the loss to *loss.
__global__ void __launch_bounds__(THREADS, 1) k_mlp_train(Net net, const float* __restrict__ feats,
                                                          const float* __restrict__ targets,
                                                          const int* __restrict__ index, int first, int rows,
                                                          float* __restrict__ grads, float* loss, int* status) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint64_t* bar = (uint64_t*)(sm + S_TRAIN_END);
    uint32_t* slot = (uint32_t*)(sm + S_TRAIN_END + 8);
    const int tid = threadIdx.x, warp = tid >> 5;
    load_view<64, 16>(sm + S_W1, net.w1t);
    load_view<64, 64>(sm + S_W2, net.w2t);
    load_view<16, 64>(sm + S_W3, net.w3t);
    load_view<64, 64>(sm + S_W2N, net.w2n);
    load_view<64, 16>(sm + S_W3N, net.w3n);
    bar_init(bar);
    const uint32_t tmem = tmem_take(slot, TRAIN_COLS);
    const uint32_t lane = (uint32_t)(warp * 32) << 16;
    const uint32_t b = saddr(bar);
    const float* b1 = net.master + O_B1;
    const float* b2 = net.master + O_B2;
    const float* b3 = net.master + O_B3;
    const float scale = 2.0f / (float)rows;
    uint32_t phase = 0;
    const int tiles = (rows + TILE - 1) / TILE;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int r = t * TILE + tid;
        const bool valid = r < rows;
        const size_t at = valid ? (size_t)(index ? index[first + r] : first + r) : 0;
        // X, and X^T with the ones row into [H1^T; X^T; 1]
#pragma unroll
        for (int j = 0; j < IN; j++) {
            const float v = valid ? (feats[at * IN + j] - net.mean[j]) * net.inv_std[j] : 0.0f;
            put(sm + S_XA, tid, j, 128, v);
            put(sm + S_AG, HID + j, tid, 128, v);
        }
        put(sm + S_AG, HID + IN, tid, 128, valid ? 1.0f : 0.0f);
        put(sm + S_A3, HID, tid, 128, valid ? 1.0f : 0.0f);
        operands_ready();
        if (tid == 0) {
            mma(tmem, operand(saddr(sm + S_XA), 128, 0), operand(saddr(sm + S_W1), 64, 0), idesc(128, 64), 0);
            commit(b);
        }
        if (!products_done(b, phase, status)) break;
        uint32_t v[64];
        tmem_ld_x64(tmem + lane, v);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < HID; j++) {
            const float h = silu(__uint_as_float(v[j]) + b1[j]);
            put(sm + S_H1, tid, j, 128, h);
            put(sm + S_AG, j, tid, 128, h);
        }
        operands_ready();
        if (tid == 0) {
            for (int s = 0; s < 4; s++)
                mma(tmem + 64, operand(saddr(sm + S_H1), 128, s), operand(saddr(sm + S_W2), 64, s), idesc(128, 64),
                    s > 0);
            commit(b);
        }
        if (!products_done(b, phase, status)) break;
        tmem_ld_x64(tmem + lane + 64, v);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < HID; j++) {
            const float h = silu(__uint_as_float(v[j]) + b2[j]);
            put(sm + S_H2, tid, j, 128, h);
            put(sm + S_A3, j, tid, 128, h);
        }
        operands_ready();
        if (tid == 0) {
            for (int s = 0; s < 4; s++)
                mma(tmem + 128, operand(saddr(sm + S_H2), 128, s), operand(saddr(sm + S_W3), 16, s),
                    idesc(128, 16), s > 0);
            commit(b);
        }
        if (!products_done(b, phase, status)) break;
        uint32_t y[16];
        tmem_ld_x16(tmem + lane + 128, y);
        tmem_wait_ld();
        // D3 = 2 (y - t) / batch: into D3 (K padded to 16) and D3^T
        float d3[OUT], sq = 0.0f;
#pragma unroll
        for (int j = 0; j < OUT; j++) {
            const float e = valid ? (__uint_as_float(y[j]) + b3[j]) - targets[at * OUT + j] : 0.0f;
            sq += e * e;
            d3[j] = scale * e;
        }
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const float d = k < OUT ? d3[k] : 0.0f;
            put(sm + S_D3, tid, k, 128, d);
            put(sm + S_B3, k, tid, 16, d);
        }
        operands_ready();
        if (tid == 0) {  // dH2 = D3 W3^T
            mma(tmem + 144, operand(saddr(sm + S_D3), 128, 0), operand(saddr(sm + S_W3N), 64, 0), idesc(128, 64), 0);
            commit(b);
        }
        if (!products_done(b, phase, status)) break;
        {
            uint32_t dh[64], z[64];
            tmem_ld_x64(tmem + lane + 144, dh);
            tmem_ld_x64(tmem + lane + 64, z);
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < HID; j++) {
                const float d = __uint_as_float(dh[j]) * silu_grad(__uint_as_float(z[j]) + b2[j]);
                put(sm + S_D2, tid, j, 128, d);
                put(sm + S_BG, j, tid, 128, d);
            }
        }
        operands_ready();
        if (tid == 0) {  // dH1 = D2 W2^T
            for (int s = 0; s < 4; s++)
                mma(tmem + 144, operand(saddr(sm + S_D2), 128, s), operand(saddr(sm + S_W2N), 64, s),
                    idesc(128, 64), s > 0);
            commit(b);
        }
        if (!products_done(b, phase, status)) break;
        {
            uint32_t dh[64], z[64];
            tmem_ld_x64(tmem + lane + 144, dh);
            tmem_ld_x64(tmem + lane, z);
            tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < HID; j++)
                put(sm + S_BG, HID + j, tid, 128, __uint_as_float(dh[j]) * silu_grad(__uint_as_float(z[j]) + b1[j]));
        }
        operands_ready();
        if (tid == 0) {  // the weight and bias gradients, K = the tile's samples
            for (int s = 0; s < 8; s++)
                mma(tmem, operand(saddr(sm + S_AG), 128, s), operand(saddr(sm + S_BG), 128, s), idesc(128, 128),
                    s > 0);
            for (int s = 0; s < 8; s++)
                mma(tmem + 128, operand(saddr(sm + S_A3), 128, s), operand(saddr(sm + S_B3), 16, s),
                    idesc(128, 16), s > 0);
            commit(b);
        }
        if (!products_done(b, phase, status)) break;
        {
            uint32_t g[64];
            // row tid of [dW2 | . ; . | dW1 ; db2 | db1]
            tmem_ld_x64(tmem + lane, g);
            tmem_wait_ld();
            if (tid < HID) {
                for (int j = 0; j < HID; j++) atomicAdd(&grads[O_W2 + tid * HID + j], __uint_as_float(g[j]));
            } else if (tid == HID + IN) {
                for (int j = 0; j < HID; j++) atomicAdd(&grads[O_B2 + j], __uint_as_float(g[j]));
            }
            tmem_ld_x64(tmem + lane + 64, g);
            tmem_wait_ld();
            if (tid >= HID && tid < HID + IN) {
                for (int j = 0; j < HID; j++) atomicAdd(&grads[O_W1 + (tid - HID) * HID + j], __uint_as_float(g[j]));
            } else if (tid == HID + IN) {
                for (int j = 0; j < HID; j++) atomicAdd(&grads[O_B1 + j], __uint_as_float(g[j]));
            }
            uint32_t g3[16];
            tmem_ld_x16(tmem + lane + 128, g3);
            tmem_wait_ld();
            if (tid < HID) {
                for (int j = 0; j < OUT; j++) atomicAdd(&grads[O_W3 + tid * OUT + j], __uint_as_float(g3[j]));
            } else if (tid == HID) {
                for (int j = 0; j < OUT; j++) atomicAdd(&grads[O_B3 + j], __uint_as_float(g3[j]));
            }
        }
        for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
        if ((tid & 31) == 0) atomicAdd(loss, sq / (float)rows);
        fence_before();
        __syncthreads();
        fence_after();
    }
    tmem_give(tmem, TRAIN_COLS);
}

// Adam on the FP32 masters (step counted from 1), then the BF16 operand views.
__global__ void k_adam(float* __restrict__ master, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ grads, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N_PARAMS) return;
    const float g = grads[i];
    const float mi = 0.9f * m[i] + 0.1f * g;
    const float vi = 0.999f * v[i] + 0.001f * g * g;
    m[i] = mi;
    v[i] = vi;
    master[i] = master[i] - lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

__global__ void k_views(const float* __restrict__ p, __nv_bfloat16* w1t, __nv_bfloat16* w2t, __nv_bfloat16* w3t,
                        __nv_bfloat16* w2n, __nv_bfloat16* w3n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < HID * IN) {  // w1t[n][k] = W1[k][n]
        const int n = i / IN, k = i % IN;
        w1t[i] = __float2bfloat16_rn(p[O_W1 + k * HID + n]);
    }
    if (i < HID * HID) {
        const int n = i / HID, k = i % HID;
        w2t[i] = __float2bfloat16_rn(p[O_W2 + k * HID + n]);  // W2^T
        w2n[i] = __float2bfloat16_rn(p[O_W2 + i]);            // W2
    }
    if (i < 16 * HID) {  // w3t[n][k] = W3[k][n], n < 2
        const int n = i / HID, k = i % HID;
        w3t[i] = __float2bfloat16_rn(n < OUT ? p[O_W3 + k * OUT + n] : 0.0f);
        const int n2 = i / 16, k2 = i % 16;  // w3n[n][k] = W3[n][k], k < 2
        w3n[i] = __float2bfloat16_rn(k2 < OUT ? p[O_W3 + n2 * OUT + k2] : 0.0f);
    }
}

}  // namespace mlp
}  // namespace vxr

using namespace vxr::mlp;

struct vxr_mlp {
    int device = 0, sms = 148;
    cudaStream_t stream = nullptr;
    std::string error;
    float *master = nullptr, *m = nullptr, *v = nullptr, *grads = nullptr, *norm = nullptr, *loss = nullptr;
    __nv_bfloat16 *w1t = nullptr, *w2t = nullptr, *w3t = nullptr, *w2n = nullptr, *w3n = nullptr;
    int* status = nullptr;
    long long step = 0;  // Adam steps taken
    std::vector<void*> allocations;
};

namespace {

int mfail(vxr_mlp* n, int code, const std::string& why) {
    if (n) n->error = why;
    return code;
}

#define MLP_CUDA(call)                                                                                     \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return mfail(net, VXR_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int malloc_n(vxr_mlp* net, T** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess)
        return mfail(net, VXR_ECUDA, "cudaMalloc");
    net->allocations.push_back(q);
    *p = (T*)q;
    return VXR_OK;
}

Net net_of(const vxr_mlp* n) {
    Net k;
    k.w1t = n->w1t;
    k.w2t = n->w2t;
    k.w3t = n->w3t;
    k.w2n = n->w2n;
    k.w3n = n->w3n;
    k.master = n->master;
    k.mean = n->norm;
    k.inv_std = n->norm + IN;
    return k;
}

int refresh_views(vxr_mlp* net) {
    k_views<<<(HID * HID + 255) / 256, 256, 0, net->stream>>>(net->master, net->w1t, net->w2t, net->w3t, net->w2n,
                                                               net->w3n);
    MLP_CUDA(cudaGetLastError());
    return VXR_OK;
}

int check_status(vxr_mlp* net) {
    int s = 0;
    MLP_CUDA(cudaMemcpyAsync(&s, net->status, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
    MLP_CUDA(cudaStreamSynchronize(net->stream));
    if (s != 0) return mfail(net, s, "a tensor-core product did not complete in time");
    return VXR_OK;
}

// One batch's gradients into net->grads (zeroed first) and its loss into net->loss.
int batch_gradients(vxr_mlp* net, const float* feats, const float* targets, const int* index, int first, int rows) {
    MLP_CUDA(cudaMemsetAsync(net->grads, 0, sizeof(float) * N_PARAMS, net->stream));
    MLP_CUDA(cudaMemsetAsync(net->loss, 0, sizeof(float), net->stream));
    const int tiles = (rows + TILE - 1) / TILE;
    const int blocks = std::max(1, std::min(tiles, net->sms));
    k_mlp_train<<<blocks, THREADS, TRAIN_SMEM, net->stream>>>(net_of(net), feats, targets, index, first, rows,
                                                              net->grads, net->loss, net->status);
    MLP_CUDA(cudaGetLastError());
    return VXR_OK;
}

}  // namespace

// The forward pass for other translation units of this library (the box world's learned warm start): rows read on
// the device (*rows_dev x rows_mult), enqueued on `stream`.
int vxr_mlp_forward_device(vxr_mlp* net, const float* feats, const int* rows_dev, int rows_mult, int rows_max,
                           float* out, cudaStream_t stream) {
    const int tiles = (rows_max + TILE - 1) / TILE;
    const int blocks = std::max(1, std::min(tiles, 2 * net->sms));
    k_mlp_forward<<<blocks, THREADS, FWD_SMEM, stream>>>(net_of(net), feats, rows_dev, rows_mult, 0, out,
                                                         net->status);
    return cudaGetLastError() == cudaSuccess ? VXR_OK : VXR_ECUDA;
}

extern "C" {

vxr_mlp* vxr_mlp_create(int32_t device, uint64_t seed, int32_t* status) {
    auto set = [&](int32_t s) {
        if (status) *status = s;
    };
    vxr_mlp* net = new vxr_mlp();
    net->device = device;
    auto bad = [&](int rc) {
        set(rc);
        vxr_mlp_destroy(net);
        return (vxr_mlp*)nullptr;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bad(VXR_ECUDA);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return bad(VXR_ECUDA);
    net->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess) return bad(VXR_ECUDA);
    int rc = 0;
    rc |= malloc_n(net, &net->master, N_PARAMS);
    rc |= malloc_n(net, &net->m, N_PARAMS);
    rc |= malloc_n(net, &net->v, N_PARAMS);
    rc |= malloc_n(net, &net->grads, N_PARAMS);
    rc |= malloc_n(net, &net->norm, 2 * IN);
    rc |= malloc_n(net, &net->loss, 1);
    rc |= malloc_n(net, &net->status, 1);
    rc |= malloc_n(net, &net->w1t, HID * IN);
    rc |= malloc_n(net, &net->w2t, HID * HID);
    rc |= malloc_n(net, &net->w3t, 16 * HID);
    rc |= malloc_n(net, &net->w2n, HID * HID);
    rc |= malloc_n(net, &net->w3n, HID * 16);
    if (rc) return bad(VXR_ECUDA);
    if (cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, TRAIN_SMEM) != cudaSuccess)
        return bad(VXR_ECUDA);
    // He-style initial weights from the seed; zero biases; identity normalisation
    std::mt19937_64 gen(seed);
    std::normal_distribution<double> normal(0.0, 1.0);
    std::vector<float> p(N_PARAMS, 0.0f);
    for (int i = 0; i < IN * HID; i++) p[O_W1 + i] = (float)(normal(gen) * std::sqrt(2.0 / IN));
    for (int i = 0; i < HID * HID; i++) p[O_W2 + i] = (float)(normal(gen) * std::sqrt(2.0 / HID));
    for (int i = 0; i < HID * OUT; i++) p[O_W3 + i] = (float)(normal(gen) * std::sqrt(1.0 / HID));
    std::vector<float> norm(2 * IN, 0.0f);
    for (int j = 0; j < IN; j++) norm[IN + j] = 1.0f;
    if (vxr_mlp_set(net, p.data(), norm.data(), norm.data() + IN) != VXR_OK) return bad(VXR_ECUDA);
    set(VXR_OK);
    return net;
}

void vxr_mlp_destroy(vxr_mlp* net) {
    if (!net) return;
    if (net->stream) cudaStreamSynchronize(net->stream);
    for (void* p : net->allocations) cudaFree(p);
    if (net->stream) cudaStreamDestroy(net->stream);
    delete net;
}

const char* vxr_mlp_error(const vxr_mlp* net) { return net ? net->error.c_str() : "no network"; }

int32_t vxr_mlp_set(vxr_mlp* net, const float* params, const float* mean16, const float* inv_std16) {
    if (!net) return VXR_EINVAL;
    cudaSetDevice(net->device);
    if (params) {
        MLP_CUDA(cudaMemcpy(net->master, params, sizeof(float) * N_PARAMS, cudaMemcpyHostToDevice));
        MLP_CUDA(cudaMemset(net->m, 0, sizeof(float) * N_PARAMS));
        MLP_CUDA(cudaMemset(net->v, 0, sizeof(float) * N_PARAMS));
        net->step = 0;
    }
    if (mean16) MLP_CUDA(cudaMemcpy(net->norm, mean16, sizeof(float) * IN, cudaMemcpyHostToDevice));
    if (inv_std16) MLP_CUDA(cudaMemcpy(net->norm + IN, inv_std16, sizeof(float) * IN, cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemset(net->status, 0, sizeof(int)));
    if (int rc = refresh_views(net)) return rc;
    MLP_CUDA(cudaStreamSynchronize(net->stream));
    return VXR_OK;
}

int32_t vxr_mlp_get(vxr_mlp* net, float* params, float* mean16, float* inv_std16) {
    if (!net) return VXR_EINVAL;
    MLP_CUDA(cudaStreamSynchronize(net->stream));
    if (params) MLP_CUDA(cudaMemcpy(params, net->master, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost));
    if (mean16) MLP_CUDA(cudaMemcpy(mean16, net->norm, sizeof(float) * IN, cudaMemcpyDeviceToHost));
    if (inv_std16) MLP_CUDA(cudaMemcpy(inv_std16, net->norm + IN, sizeof(float) * IN, cudaMemcpyDeviceToHost));
    return VXR_OK;
}

int32_t vxr_mlp_forward(vxr_mlp* net, const float* features, int32_t rows, float* out2) {
    if (!net || !features || !out2 || rows < 0) return mfail(net, VXR_EINVAL, "null argument");
    if (rows == 0) return VXR_OK;
    cudaSetDevice(net->device);
    float *f = nullptr, *o = nullptr;
    MLP_CUDA(cudaMallocAsync(&f, sizeof(float) * IN * (size_t)rows, net->stream));
    MLP_CUDA(cudaMallocAsync(&o, sizeof(float) * OUT * (size_t)rows, net->stream));
    MLP_CUDA(cudaMemcpyAsync(f, features, sizeof(float) * IN * (size_t)rows, cudaMemcpyHostToDevice, net->stream));
    const int tiles = (rows + TILE - 1) / TILE;
    k_mlp_forward<<<std::max(1, std::min(tiles, 2 * net->sms)), THREADS, FWD_SMEM, net->stream>>>(
        net_of(net), f, nullptr, 0, rows, o, net->status);
    MLP_CUDA(cudaGetLastError());
    MLP_CUDA(cudaMemcpyAsync(out2, o, sizeof(float) * OUT * (size_t)rows, cudaMemcpyDeviceToHost, net->stream));
    MLP_CUDA(cudaFreeAsync(f, net->stream));
    MLP_CUDA(cudaFreeAsync(o, net->stream));
    return check_status(net);
}

int32_t vxr_mlp_gradients(vxr_mlp* net, const float* features, const float* targets, int32_t rows, float* grads,
                          float* loss) {
    if (!net || !features || !targets || rows < 1) return mfail(net, VXR_EINVAL, "null argument");
    cudaSetDevice(net->device);
    float *f = nullptr, *t = nullptr;
    MLP_CUDA(cudaMallocAsync(&f, sizeof(float) * IN * (size_t)rows, net->stream));
    MLP_CUDA(cudaMallocAsync(&t, sizeof(float) * OUT * (size_t)rows, net->stream));
    MLP_CUDA(cudaMemcpyAsync(f, features, sizeof(float) * IN * (size_t)rows, cudaMemcpyHostToDevice, net->stream));
    MLP_CUDA(cudaMemcpyAsync(t, targets, sizeof(float) * OUT * (size_t)rows, cudaMemcpyHostToDevice, net->stream));
    if (int rc = batch_gradients(net, f, t, nullptr, 0, rows)) return rc;
    if (grads) MLP_CUDA(cudaMemcpyAsync(grads, net->grads, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost, net->stream));
    if (loss) MLP_CUDA(cudaMemcpyAsync(loss, net->loss, sizeof(float), cudaMemcpyDeviceToHost, net->stream));
    MLP_CUDA(cudaFreeAsync(f, net->stream));
    MLP_CUDA(cudaFreeAsync(t, net->stream));
    return check_status(net);
}

int32_t vxr_mlp_train(vxr_mlp* net, const float* features, const float* targets, int32_t rows, int32_t epochs,
                      int32_t batch, float lr, uint64_t seed, float* epoch_loss) {
    if (!net || !features || !targets || rows < 1 || epochs < 0 || batch < 1) return mfail(net, VXR_EINVAL, "bad argument");
    cudaSetDevice(net->device);
    // the inputs' normalisation, from the training data (host, doubles)
    std::vector<double> mean(IN, 0.0), var(IN, 0.0);
    for (int r = 0; r < rows; r++)
        for (int j = 0; j < IN; j++) mean[j] += features[(size_t)r * IN + j];
    for (int j = 0; j < IN; j++) mean[j] /= rows;
    for (int r = 0; r < rows; r++)
        for (int j = 0; j < IN; j++) {
            const double d = features[(size_t)r * IN + j] - mean[j];
            var[j] += d * d;
        }
    std::vector<float> m16(IN), s16(IN);
    for (int j = 0; j < IN; j++) {
        const double sd = std::sqrt(var[j] / rows);
        m16[j] = (float)mean[j];
        s16[j] = sd > 1e-12 ? (float)(1.0 / sd) : 1.0f;
    }
    if (int rc = vxr_mlp_set(net, nullptr, m16.data(), s16.data())) return rc;
    float *f = nullptr, *t = nullptr;
    int* index = nullptr;
    MLP_CUDA(cudaMalloc(&f, sizeof(float) * IN * (size_t)rows));
    MLP_CUDA(cudaMalloc(&t, sizeof(float) * OUT * (size_t)rows));
    MLP_CUDA(cudaMalloc(&index, sizeof(int) * (size_t)rows));
    MLP_CUDA(cudaMemcpy(f, features, sizeof(float) * IN * (size_t)rows, cudaMemcpyHostToDevice));
    MLP_CUDA(cudaMemcpy(t, targets, sizeof(float) * OUT * (size_t)rows, cudaMemcpyHostToDevice));
    std::vector<int> order(rows);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 gen(seed);
    int rc = VXR_OK;
    for (int e = 0; e < epochs && rc == VXR_OK; e++) {
        std::shuffle(order.begin(), order.end(), gen);
        if (cudaMemcpyAsync(index, order.data(), sizeof(int) * (size_t)rows, cudaMemcpyHostToDevice, net->stream) !=
            cudaSuccess) {
            rc = mfail(net, VXR_ECUDA, "index upload");
            break;
        }
        double sum = 0.0;
        int batches = 0;
        for (int first = 0; first < rows; first += batch) {
            const int n = std::min(batch, rows - first);
            rc = batch_gradients(net, f, t, index, first, n);
            if (rc) break;
            net->step++;
            const float c1 = 1.0f - std::pow(0.9f, (float)net->step), c2 = 1.0f - std::pow(0.999f, (float)net->step);
            k_adam<<<(N_PARAMS + 255) / 256, 256, 0, net->stream>>>(net->master, net->m, net->v, net->grads, lr, c1, c2);
            if ((rc = refresh_views(net))) break;
            float l = 0.0f;
            if (cudaMemcpyAsync(&l, net->loss, sizeof(float), cudaMemcpyDeviceToHost, net->stream) != cudaSuccess) {
                rc = mfail(net, VXR_ECUDA, "loss");
                break;
            }
            cudaStreamSynchronize(net->stream);
            sum += l;
            batches++;
        }
        if (rc == VXR_OK) rc = check_status(net);
        if (epoch_loss && batches) epoch_loss[e] = (float)(sum / batches);
    }
    cudaFree(f);
    cudaFree(t);
    cudaFree(index);
    return rc;
}

}  // extern "C"
