// epilogue.cuh -- the fused r^2 epilogue of the tensor-core kernels, applied
// to 32 accumulator columns (B rows) at a time as they leave TMEM.
//
// qLD's get_pairwise_ld_score (src/correlator/src/gemm_cpu.c:343-404):
// r^2 = 0 when a bit count is 0, values > 1.0001 become 123.456, 0/0 stays
// NaN.  Two evaluations (template MODE):
//   R2_EXACT      D = S*c - cA*cB is formed exactly in FP64 (every term is an
//                 integer below 2^53: the count enters FP64 through the 2^52
//                 bias trick and D is one fused multiply-add), then
//                 r^2 = (D*D) * (1/varA * 1/varB) with one rounding to FP32.
//                 No 64-bit integer arithmetic and one conversion per pair.
//   R2_REFERENCE  the reference's float/double operation sequence
//                 (qld_device.cuh: r2_reference), bit for bit.
// Per-column factors live in shared memory (filled once per tile); the
// per-row (A) factors in registers.
#pragma once

#include "qld_device.cuh"

namespace qld {
namespace epi {

// Shared-memory column factors of one tile: BN entries each of
// d0 (exact: 1/(c(S-c)); reference: 1 - c/S), d1 (exact: c as double),
// c (bit count), v (reference: c/S as float).  24 bytes per column.
struct Cols {
    double *d0, *d1;
    uint32_t *c;
    float *v;
    __device__ __forceinline__ Cols(uint8_t *base, int bn)
        : d0(reinterpret_cast<double *>(base)),
          d1(reinterpret_cast<double *>(base) + bn),
          c(reinterpret_cast<uint32_t *>(reinterpret_cast<double *>(base) + 2 * bn)),
          v(reinterpret_cast<float *>(reinterpret_cast<uint32_t *>(
                reinterpret_cast<double *>(base) + 2 * bn) + bn)) {}
};
constexpr int COL_BYTES = 24;

template <int MODE>
__device__ __forceinline__ void store_col(const Cols &f, int bl, uint32_t c, int S) {
    f.c[bl] = c;
    if (MODE == R2_EXACT) {
        f.d0[bl] = row_exact(c, S).inv_var;
        f.d1[bl] = (double)c;
    } else {
        const RowRef r = row_ref(c, S);
        f.v[bl] = r.v;
        f.d0[bl] = r.one_minus;
    }
}

// Per-thread A-row factors.
struct ARow {
    uint32_t c;
    double inv, cd;     // exact
    RowRef ref;         // reference
};

template <int MODE>
__device__ __forceinline__ ARow make_arow(uint32_t c, int S) {
    ARow r;
    r.c = c;
    if (MODE == R2_EXACT) {
        r.inv = row_exact(c, S).inv_var;
        r.cd = (double)c;
    } else {
        r.ref = row_ref(c, S);
    }
    return r;
}

__device__ __forceinline__ double u32_to_f64(uint32_t x) {
    // 2^52 + x has the integer x in its low mantissa bits; subtracting 2^52 is exact.
    return __hiloint2double(0x43300000, (int)x) - 4503599627370496.0;
}

template <int MODE>
__device__ __forceinline__ float pair_r2(uint32_t cnt, const ARow &ra, const Cols &f, int bl,
                                         double S_d, int S) {
    if (MODE == R2_EXACT) {
        const double cbd = f.d1[bl];
        const double D = fma(S_d, u32_to_f64(cnt), -(ra.cd * cbd));
        const double r = (D * D) * (ra.inv * f.d0[bl]);
        if (ra.c == 0u || cbd == 0.0) return 0.0f;
        if (r > 1.0001) return 123.456f;
        return __double2float_rn(r);
    } else {
        RowRef rb;
        rb.c = f.c[bl];
        rb.v = f.v[bl];
        rb.one_minus = f.d0[bl];
        return r2_reference(cnt, ra.ref, rb, S);
    }
}

// One 32-column chunk: accumulators v[t] (holding count << shift) of A row a
// against B rows b0 + t (local columns bl0 + t).  Output element (b, a) goes
// to r2[(b - row0) * ldr + a] (and counts likewise).  Only entries inside the
// task (b < n, a < m) and the diagonal window dlo <= a - b <= dhi are
// written (a single region: a >= b; a band: 1 <= a - b <= W).
template <int MODE, int SHIFT>
__device__ __forceinline__ void chunk(const uint32_t (&v)[32], const ARow &ra, const Cols &f,
                                      int bl0, int b0, int a, bool a_ok, int n, int dlo,
                                      int dhi, float *r2, long long ldr, uint32_t *counts,
                                      long long ldc, int row0, int S) {
    if (!a_ok) return;
    const double S_d = (double)S;
    float *o = r2 + (long long)(b0 - row0) * ldr + a;
    uint32_t *oc = counts ? counts + (long long)(b0 - row0) * ldc + a : nullptr;
    const bool interior = (b0 + 31 < n) && (a - (b0 + 31) >= dlo) && (a - b0 <= dhi);
    if (interior) {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const uint32_t cnt = v[t] >> SHIFT;
            o[(long long)t * ldr] = pair_r2<MODE>(cnt, ra, f, bl0 + t, S_d, S);
            if (oc) oc[(long long)t * ldc] = cnt;
        }
    } else {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const int b = b0 + t;
            if (b < n && a - b >= dlo && a - b <= dhi) {
                const uint32_t cnt = v[t] >> SHIFT;
                o[(long long)t * ldr] = pair_r2<MODE>(cnt, ra, f, bl0 + t, S_d, S);
                if (oc) oc[(long long)t * ldc] = cnt;
            }
        }
    }
}

}  // namespace epi
}  // namespace qld
