// rows.cu -- table rows re-pitched on the device after a host upload.
//
// The counts kernels read tables whose rows start 16-byte aligned (an even
// word pitch, for TMA), while qLD-compute's tables hold K words per row back
// to back (k = compressed_snp_size, src/correlator/src/gemm_cpu.c:432-436).
// With K odd the host copy cannot land rows in place as one 1-D copy; it goes
// to a staging buffer and this kernel spreads it to the padded pitch.
#include <cstdint>

#include <cuda_runtime.h>

#include "qld_kernels.h"

namespace qld {
namespace {

constexpr int kRowsPerBlock = 8;   // one warp per row

// dst[r * ldd + w] = src[r * K + w] for w < K, 0 for K <= w < ldd.  A warp
// moves 32 consecutive words of a row per step (coalesced on both sides).
__global__ void __launch_bounds__(32 * kRowsPerBlock)
k_pad_rows(uint64_t *__restrict__ dst, long long ldd, const uint64_t *__restrict__ src, int K,
           long long rows) {
    const long long row = (long long)blockIdx.x * kRowsPerBlock + (threadIdx.x >> 5);
    if (row >= rows) return;
    const uint64_t *s = src + row * K;
    uint64_t *d = dst + row * ldd;
    for (long long w = threadIdx.x & 31; w < ldd; w += 32) d[w] = w < K ? s[w] : 0ull;
}

}  // namespace

cudaError_t launch_pad_rows(uint64_t *dst, long long ldd, const uint64_t *src, int K,
                            long long rows, cudaStream_t st) {
    if (rows <= 0) return cudaSuccess;
    if (ldd < K || K < 1) return cudaErrorInvalidValue;
    const long long blocks = (rows + kRowsPerBlock - 1) / kRowsPerBlock;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    k_pad_rows<<<(unsigned)blocks, 32 * kRowsPerBlock, 0, st>>>(dst, ldd, src, K, rows);
    return cudaGetLastError();
}

}  // namespace qld
