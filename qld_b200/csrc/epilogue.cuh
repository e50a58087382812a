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
//                 branch-free in FP32 (r2_reference_ff) with a rare
//                 fallback to the literal sequence.
// Per-column factors live in shared memory (filled once per tile); the
// per-row (A) factors in registers.
#pragma once

#include "qld_device.cuh"

namespace qld {
namespace epi {

// ------------------------------------------- R2_REFERENCE column factors --
//
// One float4 per column (and per A row, in registers): x = v = fl32(c/S) as
// the reference computes it; y + z = 1/(v(1-v)) as an unevaluated pair of
// floats (y = RN32 of the FP64 value, z = RN32 of the remainder: ~2^-48
// relative); w = RN32(1/v).  A zero row (c = 0) is all zeros, so every pair
// with it evaluates to 0 -- the reference's rule for an empty SNP -- without
// a test.  A row with v >= 1 (c = S, or a bit count above S) carries a NaN
// in y, which sends every pair with it to the literal sequence.
struct ColsR {
    float4 *f;
    __device__ __forceinline__ ColsR(uint8_t *base, int) : f(reinterpret_cast<float4 *>(base)) {}
};
constexpr int COLR_BYTES = 16;

__device__ __forceinline__ float4 ref_factors(uint32_t c, int S) {
    if (c == 0u) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float v = __fdiv_rn((float)c, (float)S);
    if (!(v < 1.0f)) return make_float4(v, __uint_as_float(0x7FC00000u), 0.0f, 1.0f);
    const double om = __dsub_rn(1.0, (double)v);
    const double i = __ddiv_rn(1.0, __dmul_rn((double)v, om));
    const float hi = __double2float_rn(i);
    return make_float4(v, hi, __double2float_rn(__dsub_rn(i, (double)hi)), __frcp_rn(v));
}

__device__ __forceinline__ void store_col_ref(const ColsR &f, int bl, uint32_t c, int S) {
    f.f[bl] = ref_factors(c, S);
}

// Per-thread A-row factors of the reference mode.
struct ARowR {
    float4 k;           // ref_factors of the row
    uint32_t c;
    float Sf, rSf;      // (float)S and its correctly rounded reciprocal
};

__device__ __forceinline__ ARowR make_arow_ref(uint32_t c, int S) {
    ARowR r;
    r.k = ref_factors(c, S);
    r.c = c;
    r.Sf = (float)S;
    r.rSf = __frcp_rn(r.Sf);
    return r;
}

// Shared-memory column factors of one tile for the integer-count kernels:
// BN entries each of d0 = 1/(c(S-c)) and d1 = c as double (R2_EXACT), or one
// ColsR float4 at the same address (R2_REFERENCE).  24 bytes per column.
struct Cols {
    uint8_t *base;
    double *d0, *d1;
    __device__ __forceinline__ Cols(uint8_t *b, int bn)
        : base(b), d0(reinterpret_cast<double *>(b)), d1(reinterpret_cast<double *>(b) + bn) {}
};
constexpr int COL_BYTES = 24;

template <int MODE>
__device__ __forceinline__ void store_col(const Cols &f, int bl, uint32_t c, int S) {
    if (MODE == R2_EXACT) {
        f.d0[bl] = row_exact(c, S).inv_var;
        f.d1[bl] = (double)c;
    } else {
        store_col_ref(ColsR(f.base, 0), bl, c, S);
    }
}

// Per-thread A-row factors.
struct ARow {
    uint32_t c;
    double inv, cd;     // exact
    ARowR rr;           // reference
};

template <int MODE>
__device__ __forceinline__ ARow make_arow(uint32_t c, int S) {
    ARow r;
    r.c = c;
    if (MODE == R2_EXACT) {
        r.inv = row_exact(c, S).inv_var;
        r.cd = (double)c;
    } else {
        r.rr = make_arow_ref(c, S);
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
// The reference's operation sequence (r2_reference) gives, per pair,
// fl32(RN64(x / den)) with x = fl32(d*d), d = fl32(v3 - p12),
// v3 = fl32(cab/S), p12 = fl32(vA*vB) and den = RN64(RN64(p12*(1-vA))*(1-vB)).
// r2_reference_ff evaluates it in FP32 alone (no FP64 instruction, no
// conversion, no MUFU), branch-free:
//  * v3 by Markstein's FMA correction: q = RN(cab * y) with y = RN(1/S),
//    then RN(q + (cab - q*S) * y), the residual exact in one FMA; with y the
//    correctly rounded reciprocal this is the correctly rounded quotient
//    (P. Markstein, IBM J. Res. Dev. 34(1), 1990); cab and S are integers
//    <= 2^24, exact in FP32.  p12, d and x as in the reference (__f*_rn: no
//    contraction).
//  * 1/den to ~2^-45: with e = vA*vB - p12 exact (the FMA TwoProduct),
//    p12*(1-vA)*(1-vB) = vA(1-vA) * vB(1-vB) * (1 - e/(vA vB)), so
//    1/den = IA * IB * (1 + t) up to 2^-48, where IA = 1/(vA(1-vA)) and IB
//    are the rows' float pairs (y + z) and t = e * (1/vA) * (1/vB); the
//    reference's two FP64 roundings of den move it by at most 2^-52.
//    q = x * IA * IB * (1 + t) is formed as an unevaluated float pair
//    (qh, ql) with FMA products (Dekker / Ogita-Rump-Oishi style error-free
//    transformations).
//  * The rounding test: RN32(qh + ql +- 2^-40 qh) are equal when no FP32
//    rounding midpoint lies within 2^-40 of the quotient, far beyond the
//    evaluation error, and then RN32(qh + ql) = fl32(RN64(x / den)).
//    Pairs failing it (~1e-5 at realistic S; more at S <= 100, whose simple
//    fractions meet midpoints more often), with a row whose v >= 1 (NaN
//    factors), or with 0 < x < 2^-100 (a subnormal-range quotient) are
//    flagged and recomputed by r2_flagged: a fixed SNP (v = 1) from x alone,
//    the rest with r2_reference.
//  * (double)r > 1.0001 is r > 1 + 838 * 2^-23, the largest float not above
//    1.0001.
// Exact zeros need no test: a zero row's factors are 0, so q = 0.
// The earlier FP64 form (Newton reciprocal of den from rcp.approx.f64 with a
// rounding test in FP64) spent its time in FP64 conversions and the MUFU.
// fl32(cab / S) for integer cab <= S <= 2^24 (exact in FP32), by Markstein's
// correction of RN(cab * RN(1/S)): the correctly rounded quotient.
__device__ __forceinline__ float ref_quotient_ff(float cab, const ARowR &A) {
    const float q0 = __fmul_rn(cab, A.rSf);
    return __fmaf_rn(__fmaf_rn(-q0, A.Sf, cab), A.rSf, q0);
}

__device__ __forceinline__ float r2_reference_ff(float cab, const ARowR &A, float4 B,
                                                 bool &redo) {
    const float v3 = ref_quotient_ff(cab, A);
    const float p12 = __fmul_rn(A.k.x, B.x);
    const float e = __fmaf_rn(A.k.x, B.x, -p12);
    const float d = __fsub_rn(v3, p12);
    const float x = __fmul_rn(d, d);
    const float Ph = __fmul_rn(A.k.y, B.y);
    float Pl = __fmaf_rn(A.k.y, B.y, -Ph);
    Pl = __fmaf_rn(A.k.y, B.z, Pl);
    Pl = __fmaf_rn(A.k.z, B.y, Pl);
    const float t = __fmul_rn(e, __fmul_rn(A.k.w, B.w));
    const float qh = __fmul_rn(x, Ph);
    float ql = __fmaf_rn(x, Ph, -qh);
    ql = __fmaf_rn(x, Pl, ql);
    ql = __fmaf_rn(qh, t, ql);
    const float rh = __fadd_rn(qh, __fmaf_rn(qh, 0x1p-40f, ql));
    const float rl = __fadd_rn(qh, __fmaf_rn(qh, -0x1p-40f, ql));
    const bool tiny = __float_as_uint(x) - 1u < __float_as_uint(0x1p-100f) - 1u;
    redo = !(rh == rl) || tiny;
    return rh > __uint_as_float(0x3F800000u + 838u) ? 123.456f : rh;
}

// A pair the fast path flagged.  A fixed SNP (v = 1: every sample carries
// the allele) makes the reference's denominator p12 (1 - vA)(1 - vB) exactly
// +0, so its quotient is x / +0 = +inf, hence 123.456, or 0 / 0, the x86
// default NaN 0xFFC00000 (gemm_cpu.c:363-389); that needs x alone, with the
// reference's float rounding, and no FP64 division.  Empty SNPs keep the
// zero rule; bit counts above S and the rare rounding cases run the literal
// sequence.  q = fl32((float)cab / S), the reference's v3.
__device__ __forceinline__ float r2_fixed(float q, float vA, float vB) {
    const float d = __fsub_rn(q, __fmul_rn(vA, vB));
    return __fmul_rn(d, d) == 0.0f ? __uint_as_float(0xFFC00000u) : 123.456f;
}

__device__ __forceinline__ float r2_flagged(uint32_t cab, const RowRef &A, const RowRef &B,
                                            int S, float q) {
    if (A.v == 0.0f || B.v == 0.0f) return 0.0f;
    if (A.v <= 1.0f && B.v <= 1.0f && (A.v == 1.0f || B.v == 1.0f)) return r2_fixed(q, A.v, B.v);
    return r2_reference(cab, A, B, S);
}

// The reference-mode chunk of CW (<= 32) columns: every pair on the fast
// path, the flagged ones (their accumulator word kept in v, a bit in `redo`)
// redone with r2_flagged.
// FLOATCNT: v holds each count as F32 bits (the 4-bit kernels' accumulators),
// else as an integer shifted left by SHIFT.
template <int SHIFT, bool FLOATCNT, int CW = 32>
__device__ __forceinline__ void chunk_ref(uint32_t (&v)[CW], const ARowR &ra, const ColsR &f,
                                          int bl0, int b0, int a, bool a_ok, int n, int dlo,
                                          int dhi, float *r2, long long ldr, uint32_t *counts,
                                          long long ldc, int row0, int S) {
    uint32_t *oc = (counts && a_ok) ? counts + (long long)(b0 - row0) * ldc + a : nullptr;
    uint32_t redo = 0;
    if (S <= (1 << 24)) {
#pragma unroll
        for (int t = 0; t < CW; ++t) {
            const uint32_t raw = v[t];
            const float cf = FLOATCNT ? __uint_as_float(raw) : (float)(raw >> SHIFT);
            const int b = b0 + t;
            if (oc && b < n && a - b >= dlo && a - b <= dhi)
                oc[(long long)t * ldc] = FLOATCNT ? (uint32_t)cf : raw >> SHIFT;
            bool rd;
            const float r = r2_reference_ff(cf, ra, f.f[bl0 + t], rd);
            v[t] = rd ? raw : __float_as_uint(r);   // a flagged pair keeps its count
            redo |= (uint32_t)rd << t;
        }
    } else {
#pragma unroll
        for (int t = 0; t < CW; ++t) {
            const uint32_t cnt = FLOATCNT ? (uint32_t)__uint_as_float(v[t]) : v[t] >> SHIFT;
            const int b = b0 + t;
            if (oc && b < n && a - b >= dlo && a - b <= dhi) oc[(long long)t * ldc] = cnt;
        }
        redo = CW == 32 ? 0xFFFFFFFFu : (1u << CW) - 1u;
    }
    if (!a_ok) redo = 0;
    if (__any_sync(0xffffffffu, redo != 0)) {
        // A lane whose A row is a fixed SNP (v = 1) has all its pairs flagged:
        // they take r2_flagged's fixed-SNP rule here in one pass, with
        // r2_reference_ff's quotient, instead of one trip each through the
        // warp-wide loop below (columns with bit counts above S stay flagged).
        const bool a_fixed = S <= (1 << 24) && ra.k.x == 1.0f && redo != 0u;
        if (__any_sync(0xffffffffu, a_fixed) && a_fixed) {
#pragma unroll
            for (int t = 0; t < CW; ++t) {
                const float vb = f.f[bl0 + t].x;
                if (((redo >> t) & 1u) && vb <= 1.0f) {
                    const float cf = FLOATCNT ? __uint_as_float(v[t]) : (float)(v[t] >> SHIFT);
                    v[t] = __float_as_uint(
                        vb == 0.0f ? 0.0f : r2_fixed(ref_quotient_ff(cf, ra), 1.0f, vb));
                    redo &= ~(1u << t);
                }
            }
        }
        if (__any_sync(0xffffffffu, redo != 0)) {
            RowRef rA;
            rA.c = ra.c;
            rA.v = ra.k.x;
            rA.one_minus = __dsub_rn(1.0, (double)ra.k.x);
#pragma unroll
            for (int t = 0; t < CW; ++t) {
                const bool rd = (redo >> t) & 1u;
                if (__any_sync(0xffffffffu, rd) && rd) {
                    const float4 cb = f.f[bl0 + t];
                    RowRef rb;
                    rb.c = cb.x != 0.0f;        // only the zero rule reads it
                    rb.v = cb.x;
                    rb.one_minus = __dsub_rn(1.0, (double)cb.x);
                    const uint32_t cnt =
                        FLOATCNT ? (uint32_t)__uint_as_float(v[t]) : v[t] >> SHIFT;
                    const float q = S <= (1 << 24) ? ref_quotient_ff((float)cnt, ra)
                                                   : __fdiv_rn((float)cnt, (float)S);
                    v[t] = __float_as_uint(r2_flagged(cnt, rA, rb, S, q));
                }
            }
        }
    }
    if (!a_ok) return;
    float *o = r2 + (long long)(b0 - row0) * ldr + a;
    const bool interior = (b0 + CW - 1 < n) && (a - (b0 + CW - 1) >= dlo) && (a - b0 <= dhi);
    if (interior) {
#pragma unroll
        for (int t = 0; t < CW; ++t) o[(long long)t * ldr] = __uint_as_float(v[t]);
    } else {
#pragma unroll
        for (int t = 0; t < CW; ++t) {
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
        chunk_ref<SHIFT, false>(v, ra.rr, ColsR(f.base, 0), bl0, b0, a, a_ok, n, dlo, dhi, r2,
                                ldr, counts, ldc, row0, S);
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

// One chunk of CW (<= 32) columns of F32 accumulators v[t] (count c as float bits), as
// chunk<R2_EXACT, 0> with the FP32 evaluation above.  taddr is the TMEM
// address the chunk was loaded from: the rare pairs whose FP32 value lies
// above 1.00009 are re-evaluated in FP64 from their count, reloaded one
// column at a time (warp-uniform loads, off the common path).
template <int CW = 32>
__device__ __forceinline__ void chunk_f32(uint32_t (&v)[CW], uint32_t taddr, const ARowF &ra,
                                          const ColsF &f, int bl0, int b0, int a, bool a_ok,
                                          int n, int dlo, int dhi, float *r2, long long ldr,
                                          uint32_t *counts, long long ldc, int row0, int S) {
    const float S_f = (float)S;
    if (counts && a_ok) {
#pragma unroll
        for (int t = 0; t < CW; ++t) {
            const int b = b0 + t;
            if (b < n && a - b >= dlo && a - b <= dhi)
                counts[(long long)(b - row0) * ldc + a] = (uint32_t)__uint_as_float(v[t]);
        }
    }
    float rmax = 0.0f;
#pragma unroll
    for (int t = 0; t < CW; ++t) {
        const float r = pair_r2_f32(__uint_as_float(v[t]), S_f, ra, f.f[bl0 + t]);
        rmax = fmaxf(rmax, r);
        v[t] = __float_as_uint(r);
    }
    if (__any_sync(0xffffffffu, rmax > 1.00009f)) {
#pragma unroll
        for (int t = 0; t < CW; ++t) {
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
    const bool interior = (b0 + CW - 1 < n) && (a - (b0 + CW - 1) >= dlo) && (a - b0 <= dhi);
    if (interior) {
#pragma unroll
        for (int t = 0; t < CW; ++t) o[(long long)t * ldr] = __uint_as_float(v[t]);
    } else {
#pragma unroll
        for (int t = 0; t < CW; ++t) {
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
    template <int CW>
    __device__ __forceinline__ void fold(const uint32_t (&v)[CW], int b0, int a, bool a_ok,
                                         int n, int symmetric, float threshold) {
        if (!a_ok) return;
#pragma unroll
        for (int t = 0; t < CW; ++t) {
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
