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
