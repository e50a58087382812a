// mxf4_rows.cuh -- the bit -> E2M1 unpack of the SM-pair 4-bit kernels
// (ld_mxf4_pair.cu, ld_batch.cu), organised as row tasks over a CTA's packed
// A rows followed by its packed B rows.
#pragma once

#include <stdint.h>

#include "tcgen05.cuh"

namespace qld {
namespace mxf4rows {

// One unpack task: one packed row (A or B) of the CTA, both 16-byte halves
// of the 32 bytes (256 samples) a sub-stage takes from each 64-byte packed
// row.  A quarter-warp then covers 8 consecutive rows, so its 16-byte loads
// from the 64-byte-swizzled packed stage and its stores into the
// 128-byte-swizzled unpacked stage both touch all 32 banks once.
struct RowTask {
    uint32_t src, xr, is_a, valid;
    uint32_t off[8];     // destination: row base + swizzled offset of chunk 0..7
};

// Task of CTA row `row` (0..HM-1: A rows, then B rows; nrows in all).
template <int HM>
__device__ __forceinline__ RowTask make_task(int row, int nrows) {
    RowTask t;
    const bool isA = row < HM;
    const int r = isA ? row : row - HM;
    t.valid = row < nrows;
    t.is_a = isA;
    t.src = (uint32_t)(r * 64);
    t.xr = (uint32_t)((r >> 1) & 3);
#pragma unroll
    for (int c = 0; c < 8; ++c) t.off[c] = (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4));
    return t;
}

template <int T>
__device__ __forceinline__ uint4 spread4(const uint4 &w) {
    return make_uint4(tc::spread_e2m1<T>(w.x), tc::spread_e2m1<T>(w.y), tc::spread_e2m1<T>(w.z),
                      tc::spread_e2m1<T>(w.w));
}

// Sub-stage `sub` (0 or 1) of a packed stage (pa, pb) into an unpacked stage
// (ua, ub): every word's bits spread over four E2M1 words (spread_e2m1).
template <int TASKS>
__device__ __forceinline__ void unpack_rows(const RowTask (&task)[TASKS], const uint8_t *pa,
                                            const uint8_t *pb, uint8_t *ua, uint8_t *ub,
                                            int sub) {
    uint4 w[TASKS][2];
#pragma unroll
    for (int j = 0; j < TASKS; ++j)
        if (task[j].valid) {
            const uint8_t *row = (task[j].is_a ? pa : pb) + task[j].src;
#pragma unroll
            for (int h = 0; h < 2; ++h)
                w[j][h] = *reinterpret_cast<const uint4 *>(
                    row + ((((uint32_t)sub * 2 + h) ^ task[j].xr) << 4));
        }
#pragma unroll
    for (int j = 0; j < TASKS; ++j) {
        if (!task[j].valid) continue;
        uint8_t *dst = task[j].is_a ? ua : ub;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            *reinterpret_cast<uint4 *>(dst + task[j].off[h * 4 + 0]) = spread4<0>(w[j][h]);
            *reinterpret_cast<uint4 *>(dst + task[j].off[h * 4 + 1]) = spread4<1>(w[j][h]);
            *reinterpret_cast<uint4 *>(dst + task[j].off[h * 4 + 2]) = spread4<2>(w[j][h]);
            *reinterpret_cast<uint4 *>(dst + task[j].off[h * 4 + 3]) = spread4<3>(w[j][h]);
        }
    }
}

}  // namespace mxf4rows
}  // namespace qld
