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
//                 (qld_device.cuh: r2_reference), bit for bit, evaluated
//                 branch-free (r2_reference_fast) with a rare fallback.
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
    float Sf, rSf;      // reference: (float)S and its correctly rounded reciprocal
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
        r.Sf = (float)S;
        r.rSf = __frcp_rn(r.Sf);
    }
    return r;
}

__device__ __forceinline__ double u32_to_f64(uint32_t x) {
    // 2^52 + x has the integer x in its low mantissa bits; subtracting 2^52 is exact.
    return __hiloint2double(0x43300000, (int)x) - 4503599627370496.0;
}

// R2_EXACT from an integer count, in FP64.
__device__ __forceinline__ float pair_r2_exact(uint32_t cnt, const ARow &ra, const Cols &f,
                                               int bl, double S_d) {
    const double cbd = f.d1[bl];
    const double D = fma(S_d, u32_to_f64(cnt), -(ra.cd * cbd));
    const double r = (D * D) * (ra.inv * f.d0[bl]);
    if (ra.c == 0u || cbd == 0.0) return 0.0f;
    if (r > 1.0001) return 123.456f;
    return __double2float_rn(r);
}

// ------------------------------------------- R2_REFERENCE without branches --
//
// The reference's operation sequence (r2_reference) rearranged so that a
// chunk's 32 pairs run branch-free and with fewer conversions:
//  * v3 = fl32(cab / S) by Markstein's FMA correction: q = RN(cab * y) with
//    y = RN(1/S), then RN(q + (cab - q*S) * y), the residual exact in one
//    FMA.  With y the correctly rounded reciprocal this is the correctly
//    rounded quotient (P. Markstein, IBM J. Res. Dev. 34(1), 1990); cab and
//    S are integers <= 2^24, exact in FP32.
//  * fl32(RN64(x / den)), the reference's FP64 division rounded to float:
//    Newton-Raphson reciprocal of den (three steps from the rcp.approx.ftz.f64
//    seed, each squaring the relative error), q = x * y with one residual
//    correction, then a rounding test in the manner of Ziv: if q lies more
//    than 64 FP64 ulps from the nearest FP32 rounding midpoint, fl32(q) =
//    fl32(RN64(x / den)).  Pairs failing it (about 3 in 10^7 at realistic S;
//    ~10^-4 at S <= 100, whose simple fractions meet midpoints more often)
//    or whose quotient would be an FP32 subnormal or negative are flagged
//    and recomputed with r2_reference.
//  * (double)r > 1.0001 is r > 1 + 838 * 2^-23, the largest float not above
//    1.0001.  x / 0 (a fixed SNP) is +inf, hence 123.456 (-inf, kept, when
//    a bit count above S makes den -0); 0 / 0 is the x86 default NaN the
//    reference's build produces (0xFFC00000).
// Moving the FP32<->FP64 conversions to integer bit-field arithmetic and
// seeding the reciprocal from the bit pattern instead (four Newton steps)
// measured slower: 5.16 / 5.42 ms against 4.78 / 4.88 ms on the single region.
__device__ __forceinline__ double rcp_seed(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return y;
}

__device__ __forceinline__ float r2_reference_fast(float cab, const RowRef &A, uint32_t cB,
                                                   float vB, double omB, float Sf, float rSf,
                                                   bool &redo) {
    const float q0 = __fmul_rn(cab, rSf);
    const float v3 = __fmaf_rn(__fmaf_rn(-q0, Sf, cab), rSf, q0);
    const float p12 = __fmul_rn(A.v, vB);
    const float d = __fsub_rn(v3, p12);
    const float r = __fmul_rn(d, d);
    const double den = __dmul_rn(__dmul_rn((double)p12, A.one_minus), omB);
    const double x = (double)r;
    double y = rcp_seed(den), e = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        e = __fma_rn(-den, y, 1.0);
        y = __fma_rn(y, e, y);
    }
    double q = __dmul_rn(x, y);
    q = __fma_rn(__fma_rn(-q, den, x), y, q);
    const long long mid = (long long)(__double_as_longlong(q) & 0x1FFFFFFFLL) - (1LL << 28);
    const bool dz = den == 0.0;
    const bool zero = A.c == 0u || cB == 0u;
    // den is 0 or in [2^-96, 1] for consistent counts; a negative den (bit
    // counts above S) takes the plain sequence.  (Dropping the range test
    // and testing the low word alone measured 4.89 / 4.82 ms against
    // 4.78 / 4.95 ms: the single-SM kernel, the one used, runs this form
    // faster.)
    // |e| <= 2^-20 before the last Newton step leaves y within ~2^-40 of
    // 1/den whatever the seed's accuracy, which the 64-ulp margin needs
    redo = !zero && !dz &&
           (!(den > 0x1p-1000 && den < 0x1p1000) || (q != 0.0 && q < 0x1p-126) ||
            (mid >= -64 && mid <= 64) || !(fabs(e) <= 0x1p-20));
    // x / 0 is an infinity of den's sign (-0 when a bit count exceeds S)
    float f = dz ? __uint_as_float(r == 0.0f ? 0xFFC00000u
                                             : 0x7F800000u | ((uint32_t)__double2hiint(den) &
                                                              0x80000000u))
                 : __double2float_rn(q);
    if (f > __uint_as_float(0x3F800000u + 838u)) f = 123.456f;
    return zero ? 0.0f : f;
}

// The reference-mode chunk: every pair on the fast path, the flagged ones
// (their accumulator word kept in v, a bit in `redo`) redone with
// r2_reference.
// FLOATCNT: v holds each count as F32 bits (the 4-bit kernels' accumulators),
// else as an integer shifted left by SHIFT.
template <int SHIFT, bool FLOATCNT>
__device__ __forceinline__ void chunk_ref(uint32_t (&v)[32], const ARow &ra, const Cols &f,
                                          int bl0, int b0, int a, bool a_ok, int n, int dlo,
                                          int dhi, float *r2, long long ldr, uint32_t *counts,
                                          long long ldc, int row0, int S) {
    uint32_t *oc = (counts && a_ok) ? counts + (long long)(b0 - row0) * ldc + a : nullptr;
    uint32_t redo = 0;
    if (S <= (1 << 24)) {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const uint32_t raw = v[t];
            const float cf = FLOATCNT ? __uint_as_float(raw) : (float)(raw >> SHIFT);
            const int b = b0 + t;
            if (oc && b < n && a - b >= dlo && a - b <= dhi)
                oc[(long long)t * ldc] = FLOATCNT ? (uint32_t)cf : raw >> SHIFT;
            bool rd;
            const float r = r2_reference_fast(cf, ra.ref, f.c[bl0 + t], f.v[bl0 + t],
                                              f.d0[bl0 + t], ra.Sf, ra.rSf, rd);
            v[t] = rd ? raw : __float_as_uint(r);   // a flagged pair keeps its count
            redo |= (uint32_t)rd << t;
        }
    } else {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const uint32_t cnt = FLOATCNT ? (uint32_t)__uint_as_float(v[t]) : v[t] >> SHIFT;
            const int b = b0 + t;
            if (oc && b < n && a - b >= dlo && a - b <= dhi) oc[(long long)t * ldc] = cnt;
        }
        redo = 0xFFFFFFFFu;
    }
    if (!a_ok) redo = 0;
    if (__any_sync(0xffffffffu, redo != 0)) {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const bool rd = (redo >> t) & 1u;
            if (__any_sync(0xffffffffu, rd) && rd) {
                RowRef rb;
                rb.c = f.c[bl0 + t];
                rb.v = f.v[bl0 + t];
                rb.one_minus = f.d0[bl0 + t];
                const uint32_t cnt = FLOATCNT ? (uint32_t)__uint_as_float(v[t]) : v[t] >> SHIFT;
                v[t] = __float_as_uint(r2_reference(cnt, ra.ref, rb, S));
            }
        }
    }
    if (!a_ok) return;
    float *o = r2 + (long long)(b0 - row0) * ldr + a;
    const bool interior = (b0 + 31 < n) && (a - (b0 + 31) >= dlo) && (a - b0 <= dhi);
    if (interior) {
#pragma unroll
        for (int t = 0; t < 32; ++t) o[(long long)t * ldr] = __uint_as_float(v[t]);
    } else {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const int b = b0 + t;
            if (b < n && a - b >= dlo && a - b <= dhi) o[(long long)t * ldr] = __uint_as_float(v[t]);
        }
    }
}

// One 32-column chunk: accumulators v[t] (holding count << shift) of A row a
// against B rows b0 + t (local columns bl0 + t).  Output element (b, a) goes
// to r2[(b - row0) * ldr + a] (and counts likewise).  Only entries inside the
// task (b < n, a < m) and the diagonal window dlo <= a - b <= dhi are
// written (a single region: a >= b; a band: 1 <= a - b <= W).
template <int MODE, int SHIFT>
__device__ __forceinline__ void chunk(uint32_t (&v)[32], const ARow &ra, const Cols &f,
                                      int bl0, int b0, int a, bool a_ok, int n, int dlo,
                                      int dhi, float *r2, long long ldr, uint32_t *counts,
                                      long long ldc, int row0, int S) {
    if constexpr (MODE == R2_REFERENCE) {
        chunk_ref<SHIFT, false>(v, ra, f, bl0, b0, a, a_ok, n, dlo, dhi, r2, ldr, counts, ldc,
                                row0, S);
    } else {
        if (!a_ok) return;
        const double S_d = (double)S;
        float *o = r2 + (long long)(b0 - row0) * ldr + a;
        uint32_t *oc = counts ? counts + (long long)(b0 - row0) * ldc + a : nullptr;
        const bool interior = (b0 + 31 < n) && (a - (b0 + 31) >= dlo) && (a - b0 <= dhi);
        if (interior) {
#pragma unroll
            for (int t = 0; t < 32; ++t) {
                const uint32_t cnt = v[t] >> SHIFT;
                o[(long long)t * ldr] = pair_r2_exact(cnt, ra, f, bl0 + t, S_d);
                if (oc) oc[(long long)t * ldc] = cnt;
            }
        } else {
#pragma unroll
            for (int t = 0; t < 32; ++t) {
                const int b = b0 + t;
                if (b < n && a - b >= dlo && a - b <= dhi) {
                    const uint32_t cnt = v[t] >> SHIFT;
                    o[(long long)t * ldr] = pair_r2_exact(cnt, ra, f, bl0 + t, S_d);
                    if (oc) oc[(long long)t * ldc] = cnt;
                }
            }
        }
    }
}

// ------------------------------------------------ 4-bit kernels, R2_EXACT --
//
// The 4-bit kernels' accumulators hold each count as an exact F32 integer
// (below 2^24, as are S, cA and cB), so D = S*c - cA*cB can be evaluated in
// FP32 with a tight bound: split cA*cB = hi + lo exactly (hi = fl(cA*cB),
// lo = fma(cA, cB, -hi), the FMA TwoProduct; lo is an integer, |lo| <= 2^23),
// then D = fl(fl(S*c - hi) - lo) with S*c - hi rounded once by an FMA.  If
// |S*c - hi| < 2^24 the FMA is exact and D is rounded once; otherwise
// |D| >= |S*c - hi| / 2 and D carries at most 3 * 2^-24 relative error.  Then r^2 = (D*D) * (invA*invB) with
// invA = fl(1/(cA(S-cA))) rounded from FP64: at most 11 * 2^-24 (6.6e-7)
// relative error against the FP64 value, a dozen FP32 instructions per pair
// instead of a chain of FP64 ones.  Exact zeros (D = 0), the 0 rule for
// empty SNPs and NaN for 0/0 match the FP64 evaluation; values above 1.00009
// (possible only when the bit counts do not match the data) are re-evaluated
// in FP64 so the 123.456 rule decides exactly as in the other kernels.
struct ColsF {
    float2 *f;   // (cB as float, 1/(cB(S-cB)) rounded to float) per column
    __device__ __forceinline__ ColsF(uint8_t *base, int) : f(reinterpret_cast<float2 *>(base)) {}
};

__device__ __forceinline__ double inv_var64(double c, double S) { return 1.0 / (c * (S - c)); }

__device__ __forceinline__ void store_col_f32(const ColsF &f, int bl, uint32_t c, int S) {
    f.f[bl] = make_float2((float)c, __double2float_rn(inv_var64((double)c, (double)S)));
}

struct ARowF {
    float ca, inv;
    bool zero;
};

__device__ __forceinline__ ARowF make_arow_f32(uint32_t c, int S) {
    ARowF r;
    r.ca = (float)c;
    r.inv = __double2float_rn(inv_var64((double)c, (double)S));
    r.zero = c == 0u;
    return r;
}

__device__ __forceinline__ float pair_r2_f32(float c, float S_f, const ARowF &ra, float2 col) {
    const float hi = __fmul_rn(ra.ca, col.x);
    const float lo = __fmaf_rn(ra.ca, col.x, -hi);
    const float D = __fsub_rn(__fmaf_rn(S_f, c, -hi), lo);
    const float r = __fmul_rn(__fmul_rn(D, D), __fmul_rn(ra.inv, col.y));
    return (ra.zero || col.x == 0.0f) ? 0.0f : r;
}

// The FP64 evaluation (pair_r2_exact) from the same exact inputs.
__device__ __forceinline__ float pair_r2_f64(float c, float ca, float cb, int S) {
    if (ca == 0.0f || cb == 0.0f) return 0.0f;
    const double Sd = (double)S, a = (double)ca, b = (double)cb;
    const double D = fma(Sd, (double)c, -(a * b));
    const double r = (D * D) * (inv_var64(a, Sd) * inv_var64(b, Sd));
    if (r > 1.0001) return 123.456f;
    return __double2float_rn(r);
}

// One 32-column chunk of F32 accumulators v[t] (count c as float bits), as
// chunk<R2_EXACT, 0> with the FP32 evaluation above.  taddr is the TMEM
// address the chunk was loaded from: the rare pairs whose FP32 value lies
// above 1.00009 are re-evaluated in FP64 from their count, reloaded one
// column at a time (warp-uniform loads, off the common path).
__device__ __forceinline__ void chunk_f32(uint32_t (&v)[32], uint32_t taddr, const ARowF &ra,
                                          const ColsF &f, int bl0, int b0, int a, bool a_ok,
                                          int n, int dlo, int dhi, float *r2, long long ldr,
                                          uint32_t *counts, long long ldc, int row0, int S) {
    const float S_f = (float)S;
    if (counts && a_ok) {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const int b = b0 + t;
            if (b < n && a - b >= dlo && a - b <= dhi)
                counts[(long long)(b - row0) * ldc + a] = (uint32_t)__uint_as_float(v[t]);
        }
    }
    float rmax = 0.0f;
#pragma unroll
    for (int t = 0; t < 32; ++t) {
        const float r = pair_r2_f32(__uint_as_float(v[t]), S_f, ra, f.f[bl0 + t]);
        rmax = fmaxf(rmax, r);
        v[t] = __float_as_uint(r);
    }
    if (__any_sync(0xffffffffu, rmax > 1.00009f)) {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const bool redo = __uint_as_float(v[t]) > 1.00009f;
            if (__any_sync(0xffffffffu, redo)) {
                uint32_t w;
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];"
                             : "=r"(w)
                             : "r"(taddr + (uint32_t)t));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (redo)
                    v[t] = __float_as_uint(
                        pair_r2_f64(__uint_as_float(w), ra.ca, f.f[bl0 + t].x, S));
            }
        }
    }
    if (!a_ok) return;
    float *o = r2 + (long long)(b0 - row0) * ldr + a;
    const bool interior = (b0 + 31 < n) && (a - (b0 + 31) >= dlo) && (a - b0 <= dhi);
    if (interior) {
#pragma unroll
        for (int t = 0; t < 32; ++t) o[(long long)t * ldr] = __uint_as_float(v[t]);
    } else {
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const int b = b0 + t;
            if (b < n && a - b >= dlo && a - b <= dhi) o[(long long)t * ldr] = __uint_as_float(v[t]);
        }
    }
}

// A warp's share of a task summary (BatchSummary): fold() takes the r^2
// values chunk_f32 left in v (A row a against B rows b0 + t), flush() sums
// the warp's lanes and adds them to the task's summary with three atomics.
struct SumAcc {
    double sum = 0.0;
    unsigned long long cnt = 0;
    float mx = 0.0f;
    __device__ __forceinline__ void fold(const uint32_t (&v)[32], int b0, int a, bool a_ok,
                                         int n, int symmetric, float threshold) {
        if (!a_ok) return;
#pragma unroll
        for (int t = 0; t < 32; ++t) {
            const int b = b0 + t;
            const float r = __uint_as_float(v[t]);
            // a pair of the task, and not NaN or the 123.456 sentinel
            if (b < n && (!symmetric || a > b) && r < 100.0f) {
                sum += (double)r;
                cnt += r >= threshold;
                mx = fmaxf(mx, r);
            }
        }
    }
    __device__ __forceinline__ void flush(BatchSummary *out) {
        for (int o = 16; o > 0; o >>= 1) {
            sum += __shfl_down_sync(0xffffffffu, sum, o);
            cnt += __shfl_down_sync(0xffffffffu, cnt, o);
            mx = fmaxf(mx, __shfl_down_sync(0xffffffffu, mx, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&out->sum, sum);
            atomicAdd(&out->n_above, cnt);
            atomicMax(&out->max_bits, __float_as_uint(mx));
        }
    }
};

}  // namespace epi
}  // namespace qld
