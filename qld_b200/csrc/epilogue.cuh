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

// The FP64 evaluation (pair_r2<R2_EXACT>) from the same exact inputs.
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
