// qld_device.cuh -- device-side building blocks shared by the counts kernels:
// launch parameters, mbarrier / TMA wrappers with bounded waits, and the two
// fused r^2 epilogues.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace qld {

// Bits of the per-context device status word.  A kernel that gives up a
// bounded wait sets one and returns; the host turns it into QLD_ERR_TIMEOUT.
enum : unsigned {
    ST_TIMEOUT_FULL = 1u,    // consumer waited too long for a TMA stage
    ST_TIMEOUT_EMPTY = 2u,   // producer waited too long for a free stage
    ST_TIMEOUT_DRAIN = 4u,   // copies still in flight at exit
    ST_TIMEOUT_MMA = 8u,     // tensor-core commit never arrived
    ST_TIMEOUT_UNPACK = 16u, // unpack stage handshake timed out
};

enum R2Mode : int { R2_EXACT = 0, R2_REFERENCE = 1 };

// One launch of a counts kernel: tile (ta, tb) covers A rows
// [ta*BM, ta*BM+BM) and B rows [tb*BN, tb*BN+BN); blockIdx.y + tb0 = tb.
struct LdParams {
    int m, n, K, S;
    int symmetric;            // only entries with a >= b are produced
    int band;                 // > 0: only entries with 1 <= a - b <= band (single region)
    int tb0;                  // first B tile of this launch
    int nk;                   // K chunks (of the kernel's chunk width)
    const uint32_t *bcA, *bcB;
    float *r2;                // r2[(b - out_row0) * ldr + a]
    uint32_t *counts;         // optional, same indexing with ldc
    long long ldr, ldc;
    int out_row0;
    unsigned *status;
    long long timeout_cycles;
};

// Per-task summary a batched launch folds into its epilogue (R2_EXACT):
// over the task's pairs (a > b in a single region, all of them for two
// regions), the r^2 values below 100 (NaN and the 123.456 sentinel left
// out): their sum, how many reach the threshold, and the largest as float
// bits (r^2 >= 0, so bit order is value order).  Zeroed before the launch.
struct BatchSummary {
    double sum;
    unsigned long long n_above;
    unsigned int max_bits;
    unsigned int pad;
};

// ------------------------------------------------------------- PTX wrappers --

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

// try_wait with a suspend-time hint: the thread is parked in hardware until
// the phase completes or ~hint_ns pass, so waiting warps do not spin on the
// issue slots.
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity,
                                              uint32_t hint_ns = 20000u) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete, for at most `limit`
// SM clock cycles.  Also gives up as soon as another CTA has recorded an
// error in *status, so one failure ends the whole grid quickly.  Returns
// false when the wait was abandoned.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit,
                                          const unsigned *status) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    // Each try_wait parks the thread for up to its hint, so the clock and the
    // status word are looked at on every return.
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (clock64() - t0 > limit) return false;
        if (status && *((volatile const unsigned *)status) != 0u) return false;
    }
}

// Budget of the teardown waits: a kernel waits this long (~2 s at boost
// clock) for its own TMA copies and MMAs still in flight before it releases
// shared memory or TMEM, whatever budget its pipeline waits were given, so a
// short pipeline budget (QLD_TIMEOUT_CYCLES) never retires a CTA with work
// in flight.
constexpr long long kDrainCycles = 4000000000LL;

__device__ __forceinline__ bool grid_failed(const unsigned *status) {
    return status && *((volatile const unsigned *)status) != 0u;
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *tm) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tm)) : "memory");
}

// 2-D tiled TMA load (no multicast): box at (c0 = inner element, c1 = row)
// into shared memory, completing `bytes` on the mbarrier.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *tm, int c0, int c1,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void flag_error(unsigned *status, unsigned bit) {
    if (status) atomicOr(status, bit);
}

// ------------------------------------------------------------ r^2 epilogue --

// Per-row quantities of the epilogue, computed once per row a thread owns.
struct RowExact {
    uint32_t c;
    double inv_var;   // 1 / (c (S - c)); +inf for a monomorphic-ALT row
};

__device__ __forceinline__ RowExact row_exact(uint32_t c, int S) {
    RowExact r;
    r.c = c;
    const long long v = (long long)c * ((long long)S - (long long)c);
    r.inv_var = 1.0 / (double)v;
    return r;
}

// Exact-D r^2: D = S*cAB - cA*cB in integers, D^2 * 1/varA * 1/varB in FP64,
// one rounding to FP32.  Special cases follow gemm_cpu.c:357-389.
__device__ __forceinline__ float r2_exact(uint32_t cab, const RowExact &A, const RowExact &B,
                                          int S) {
    if (A.c == 0u || B.c == 0u) return 0.0f;
    const long long D = (long long)S * (long long)cab - (long long)A.c * (long long)B.c;
    const double d = (double)D;
    const double r = (d * d) * (A.inv_var * B.inv_var);
    if (r > 1.0001) return 123.456f;
    return __double2float_rn(r);
}

struct RowRef {
    uint32_t c;
    float v;          // (float)c / S
    double one_minus; // 1.0 - (double)v
};

__device__ __forceinline__ RowRef row_ref(uint32_t c, int S) {
    RowRef r;
    r.c = c;
    r.v = __fdiv_rn((float)c, (float)S);
    r.one_minus = __dsub_rn(1.0, (double)r.v);
    return r;
}

// get_pairwise_ld_score() (gemm_cpu.c:357-389) operation by operation:
// the intrinsics pin every rounding (no contraction into FMA), which is what
// the reference's gcc build computes.
__device__ __forceinline__ float r2_reference(uint32_t cab, const RowRef &A, const RowRef &B,
                                              int S) {
    if (B.c == 0u || A.c == 0u) return 0.0f;
    const float v3 = __fdiv_rn((float)cab, (float)S);
    const float p12 = __fmul_rn(A.v, B.v);
    const float d = __fsub_rn(v3, p12);
    float r = __fmul_rn(d, d);
    const double den = __dmul_rn(__dmul_rn((double)p12, A.one_minus), B.one_minus);
    r = __double2float_rn(__ddiv_rn((double)r, den));
    if ((double)r > 1.0001) r = 123.456f;
    return r;
}

}  // namespace qld
