// probe.cu -- self-measurement of the popcount pipe, the denominator of the
// popc variant's roofline.  Every thread keeps 8 + 8 words in registers and
// does AND + POPC on all 64 pairs per iteration (one word of each pair is
// bumped per iteration so nothing is loop-invariant); one POPC of an ANDed
// 32-bit word counts as 32 bit-ops.  The kernel touches no memory in its loop.
#include <cuda_runtime.h>
#include <stdint.h>

#include "qld_cuda.h"

namespace {

__global__ void __launch_bounds__(256) k_popc_peak(const uint32_t *seed, uint32_t *sink, int iters) {
    uint32_t a[8], b[8], acc = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        a[i] = seed[(threadIdx.x + i) & 63] ^ (blockIdx.x * 0x9E3779B9u);
        b[i] = seed[(threadIdx.x * 3 + i) & 63] + threadIdx.x;
    }
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; j += 2)
                acc += __popc(a[i] & b[j]) + __popc(a[i] & b[j + 1]);
#pragma unroll
        for (int j = 0; j < 8; ++j) b[j] += 0x01000193u;
    }
    if (acc == 0xFFFFFFFFu) sink[blockIdx.x] = acc;  // keeps the loop alive
}

}  // namespace

extern "C" int qld_cuda_measure_popc_peak(qld_ctx *ctx, double *bitops_per_s) {
    if (!ctx || !bitops_per_s) return QLD_ERR_INVALID;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return QLD_ERR_CUDA;
    uint32_t *d = nullptr;
    if (cudaMalloc(&d, 64 * 4 + 4096 * 4) != cudaSuccess) return QLD_ERR_NOMEM;
    uint32_t h[64];
    for (int i = 0; i < 64; ++i) h[i] = 0x9E3779B9u * (i + 1);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = QLD_OK;
    const int blocks = sms * 8, iters = 4096;
    if (cudaMemcpy(d, h, sizeof h, cudaMemcpyHostToDevice) != cudaSuccess) rc = QLD_ERR_CUDA;
    float best = 1e30f;
    for (int rep = 0; rep < 4 && rc == QLD_OK; ++rep) {
        cudaEventRecord(e0);
        k_popc_peak<<<blocks, 256>>>(d, d + 64, iters);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = QLD_ERR_CUDA; break; }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;   // first launch is warm-up
    }
    if (rc == QLD_OK) {
        const double popcs = (double)blocks * 256 * (double)iters * 64;
        *bitops_per_s = popcs * 32.0 / (best * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    return rc;
}

// ---------------------------------------------------------------- MMA peak --
//
// Self-measurement of the tensor pipe for the two MMA kinds the counts
// kernels issue: one CTA per SM, one thread issuing back-to-back 128 x 256
// MMAs (kind::i8, K = 32; kind::mxf4, K = 64 with 1.0 scale factors) on a
// fixed shared-memory tile into one TMEM accumulator, as the kernels do, with
// no unpack and no epilogue.  The wait for the last MMA is bounded.
#include "qld_device.cuh"
#include "tcgen05.cuh"

namespace {

using namespace qld;
using namespace qld::tc;

template <int KIND>   // 0: kind::i8, 1: kind::mxf4
__global__ void __launch_bounds__(128, 1)
k_mma_peak(int iters, unsigned *status, long long timeout) {
    extern __shared__ uint8_t raw[];
    uint8_t *sm = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 49152);
    uint32_t *slot = reinterpret_cast<uint32_t *>(sm + 49152 + 16);
    const int tid = threadIdx.x, warp = tid >> 5;
    // operands: a fixed, non-zero pattern (every E2M1 code is finite)
    for (int i = tid; i < 49152 / 4; i += 128)
        reinterpret_cast<uint32_t *>(sm)[i] = 0x9E3779B9u * (uint32_t)(i + 1);
    if (tid == 0) {
        mbar_init(smem_u32(bar), 1);
        fence_barrier_init();
    }
    fence_proxy_async_smem();
    if (warp == 0) {
        tmem_alloc<1>(smem_u32(slot), 512);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    if (KIND == 1)   // scale factors 1.0 at columns 256-271, one lane quarter per warp
        tc_st_32x32b_x16_fill(tmem + ((uint32_t)(warp * 32) << 16) + 256, 0x7F7F7F7Fu);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
        const uint32_t a0 = smem_u32(sm), b0 = smem_u32(sm + 16384);
        for (int i = 0; i < iters; ++i)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint32_t acc = (i > 0 || kk > 0) ? 1u : 0u;
                if (KIND == 0)
                    tc_mma_i8(tmem, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32),
                              idesc_i8(128, 256), acc);
                else
                    tc_mma_mxf4(tmem, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32),
                                idesc_mxf4(128, 256), acc, tmem + 256, tmem + 256);
            }
        tc_commit(smem_u32(bar));
        if (!mbar_wait(smem_u32(bar), 0, timeout, status)) flag_error(status, ST_TIMEOUT_MMA);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc<1>(tmem, 512);
    }
}

}  // namespace

extern "C" int qld_cuda_measure_mma_peak(qld_ctx *ctx, int kernel, double *ops_per_s) {
    if (!ctx || !ops_per_s || (kernel != QLD_KERNEL_MMA && kernel != QLD_KERNEL_FP4))
        return QLD_ERR_INVALID;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return QLD_ERR_CUDA;
    unsigned *status = nullptr;
    if (cudaMalloc(&status, sizeof(unsigned)) != cudaSuccess) return QLD_ERR_NOMEM;
    cudaMemset(status, 0, sizeof(unsigned));
    const int smem = 49152 + 64 + 1024, iters = 4096;
    auto kern = kernel == QLD_KERNEL_FP4 ? k_mma_peak<1> : k_mma_peak<0>;
    int rc = QLD_OK;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess)
        rc = QLD_ERR_CUDA;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4 && rc == QLD_OK; ++rep) {
        cudaEventRecord(e0);
        kern<<<sms, 128, smem>>>(iters, status, 4000000000LL);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = QLD_ERR_CUDA; break; }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    unsigned st = 0;
    if (rc == QLD_OK && cudaMemcpy(&st, status, sizeof st, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = QLD_ERR_CUDA;
    if (rc == QLD_OK && st) rc = QLD_ERR_TIMEOUT;
    if (rc == QLD_OK) {
        const double k = kernel == QLD_KERNEL_FP4 ? 64.0 : 32.0;
        *ops_per_s = 2.0 * 128 * 256 * k * 4.0 * iters * sms / (best * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(status);
    return rc;
}
