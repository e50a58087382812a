// hits.cu -- on-device r2limit filtering of a block of r^2 rows: the pairs
// qLD's report prints (writeResults, src/correlator/src/correlate_IO.c:
// 403-409: r2limit <= r^2 < 100, and for a single region only j > i) as a
// bit mask per row plus the passing values packed in report order.
//
// Three launches per block, each HBM-bound:
//   k_hits_mask     one warp per row reads the row's r^2 as float4 (128
//                   columns per warp step), writes 32-column mask words and
//                   the row's hit count;
//   k_hits_scan     one CTA: exclusive prefix of the row counts -> offsets;
//   k_hits_compact  one warp per row re-reads only the 128-column groups
//                   whose mask is not empty and writes the passing values
//                   at offset + warp prefix.
// Algorithmic bytes: rows x m x 4 read once (mask) + the non-empty groups
// again + mask and values written.
#include <cstdint>

#include "qld_kernels.h"

namespace qld {
namespace {

constexpr int kWarpsPerCta = 8;

// Predicate nibble of the 4 columns c0..c0+3 a lane holds.
__device__ __forceinline__ uint32_t nibble(const float4 &v, int c0, int lo, int m, float lim) {
    const float x[4] = {v.x, v.y, v.z, v.w};
    uint32_t nb = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int c = c0 + k;
        const bool p = c >= lo && c < m && x[k] >= lim && x[k] < 100.0f;
        nb |= (uint32_t)p << k;
    }
    return nb;
}

__global__ void __launch_bounds__(kWarpsPerCta * 32)
k_hits_mask(const float *__restrict__ r2, long long ldr, int rows, int m, int row0, int triangle,
            float lim, uint32_t *__restrict__ mask, int W, long long *__restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int r = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
    if (r >= rows) return;
    const float *row = r2 + (long long)r * ldr;
    uint32_t *mrow = mask + (long long)r * W;
    const int lo = triangle ? row0 + r + 1 : 0;
    // 128-column groups left of `lo` hold nothing that passes
    const int g_first = lo >= m ? (m + 127) / 128 : lo / 128;
    const int groups = (m + 127) / 128;
    for (int g = lane; g < g_first * 4 && g < W; g += 32) mrow[g] = 0u;
    unsigned total = 0;
    int g = g_first;
    for (; g + 1 < groups; g += 2) {
        const float4 v0 = *reinterpret_cast<const float4 *>(row + g * 128 + lane * 4);
        const float4 v1 = *reinterpret_cast<const float4 *>(row + g * 128 + 128 + lane * 4);
        uint32_t x0 = nibble(v0, g * 128 + lane * 4, lo, m, lim) << (4 * (lane & 7));
        uint32_t x1 = nibble(v1, g * 128 + 128 + lane * 4, lo, m, lim) << (4 * (lane & 7));
#pragma unroll
        for (int s = 1; s < 8; s <<= 1) {
            x0 |= __shfl_xor_sync(0xffffffffu, x0, s);
            x1 |= __shfl_xor_sync(0xffffffffu, x1, s);
        }
        if ((lane & 7) == 0) {
            const int w = g * 4 + (lane >> 3);
            if (w < W) mrow[w] = x0;
            if (w + 4 < W) mrow[w + 4] = x1;
            total += __popc(x0) + __popc(x1);
        }
    }
    if (g < groups) {
        const float4 v0 = *reinterpret_cast<const float4 *>(row + g * 128 + lane * 4);
        uint32_t x0 = nibble(v0, g * 128 + lane * 4, lo, m, lim) << (4 * (lane & 7));
#pragma unroll
        for (int s = 1; s < 8; s <<= 1) x0 |= __shfl_xor_sync(0xffffffffu, x0, s);
        if ((lane & 7) == 0) {
            const int w = g * 4 + (lane >> 3);
            if (w < W) mrow[w] = x0;
            total += __popc(x0);
        }
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) total += __shfl_xor_sync(0xffffffffu, total, s);
    if (lane == 0) cnt[r] = (long long)total;
}

// Exclusive prefix of cnt[0..rows) into off[0..rows], off[rows] = total.
__global__ void __launch_bounds__(1024) k_hits_scan(const long long *__restrict__ cnt, int rows,
                                                    long long *__restrict__ off) {
    __shared__ long long warp_sum[32];
    const int t = threadIdx.x;
    const int per = (rows + 1023) / 1024;
    const int r0 = t * per, r1 = r0 + per < rows ? r0 + per : rows;
    long long s = 0;
    for (int r = r0; r < r1; ++r) s += cnt[r];
    // inclusive scan of s over the block
    long long x = s;
    const int lane = t & 31, wid = t >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        long long w = warp_sum[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w += y;
        }
        warp_sum[lane] = w;
    }
    __syncthreads();
    long long base = x - s + (wid > 0 ? warp_sum[wid - 1] : 0);
    for (int r = r0; r < r1; ++r) {
        off[r] = base;
        base += cnt[r];
    }
    if (t == 1023) off[rows] = warp_sum[31];
}

__global__ void __launch_bounds__(kWarpsPerCta * 32)
k_hits_compact(const float *__restrict__ r2, long long ldr, int rows, int m,
               const uint32_t *__restrict__ mask, int W, const long long *__restrict__ off,
               float *__restrict__ val) {
    const int lane = threadIdx.x & 31;
    const int r = blockIdx.x * kWarpsPerCta + (threadIdx.x >> 5);
    if (r >= rows) return;
    const float *row = r2 + (long long)r * ldr;
    const uint32_t *mrow = mask + (long long)r * W;
    long long pos = off[r];
    const int groups = (m + 127) / 128;
    for (int g = 0; g < groups; ++g) {
        const int w = g * 4 + (lane >> 3);
        const uint32_t word = w < W ? mrow[w] : 0u;
        const uint32_t nb = (word >> (4 * (lane & 7))) & 0xFu;
        if (!__any_sync(0xffffffffu, nb != 0u)) continue;
        const float4 v = *reinterpret_cast<const float4 *>(row + g * 128 + lane * 4);
        const int k = __popc(nb);
        int pre = k;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, pre, d);
            if (lane >= d) pre += y;
        }
        const int tot = __shfl_sync(0xffffffffu, pre, 31);
        long long o = pos + pre - k;
        const float x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (nb >> q & 1u) val[o++] = x[q];
        pos += tot;
    }
}

}  // namespace

cudaError_t launch_hits(const float *r2, long long ldr, int rows, int m, int row0, int triangle,
                        float r2limit, uint32_t *mask, int W, long long *cnt, long long *off,
                        float *val, cudaStream_t st) {
    if (rows <= 0) return cudaSuccess;
    const int ctas = (rows + kWarpsPerCta - 1) / kWarpsPerCta;
    k_hits_mask<<<ctas, kWarpsPerCta * 32, 0, st>>>(r2, ldr, rows, m, row0, triangle, r2limit,
                                                    mask, W, cnt);
    k_hits_scan<<<1, 1024, 0, st>>>(cnt, rows, off);
    k_hits_compact<<<ctas, kWarpsPerCta * 32, 0, st>>>(r2, ldr, rows, m, mask, W, off, val);
    return cudaGetLastError();
}

}  // namespace qld
