/* CPU check of the branch-free reference-mode r^2 of the GPU epilogue
 * (qld_b200/csrc/epilogue.cuh: r2_reference_fast) against the reference's
 * operation sequence (qLD src/correlator/src/gemm_cpu.c:357-389), bit for
 * bit, over random pairs: small and large sample counts, fixed and
 * monomorphic SNPs, near-independence counts, bit counts above S.  The same steps in C: the
 * Markstein-corrected FP32 quotient cab/S, a Newton reciprocal of the FP64
 * denominator from a seed carrying an injected relative error up to 2^-8
 * (standing in for rcp.approx.ftz.f64), the residual-corrected quotient,
 * the rounding test and its fallback.  Build with -ffp-contract=off so the
 * reference sequence is not fused.
 *   usage: ref_fastpath_check N_PAIRS      exit 0 iff every pair matches */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t s_rng = 0x9E3779B97F4A7C15ull;
static uint64_t rnd(void) { s_rng ^= s_rng << 13; s_rng ^= s_rng >> 7; s_rng ^= s_rng << 17; return s_rng; }
static double urand(void) { return (double)(rnd() >> 11) * (1.0 / 9007199254740992.0); }
static uint32_t f2b(float f) { uint32_t b; memcpy(&b, &f, 4); return b; }
static float b2f(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }
static uint64_t d2b(double d) { uint64_t b; memcpy(&b, &d, 8); return b; }

static float ref_r2(uint32_t cab, uint32_t ca, uint32_t cb, int S) {
    if (ca == 0 || cb == 0) return 0.0f;
    volatile float v1 = (float)ca / (float)S, v2 = (float)cb / (float)S, v3 = (float)cab / (float)S;
    volatile float p = v1 * v2;
    volatile float d = v3 - p;
    volatile float r = d * d;
    volatile double den = (double)p * (1.0 - (double)v1) * (1.0 - (double)v2);
    r = (float)((double)r / den);
    if ((double)r > 1.0001) r = 123.456f;
    return r;
}

static float quot(float a, float S, float rS) {   /* Markstein */
    float q = a * rS;
    return fmaf(fmaf(-q, S, a), rS, q);
}

static long long fallbacks = 0;
static float fast_r2(uint32_t cab, uint32_t ca, uint32_t cb, int S, double seed_err) {
    const float Sf = (float)S, rSf = 1.0f / Sf;
    const float v1 = quot((float)ca, Sf, rSf), v2 = quot((float)cb, Sf, rSf);
    const float v3 = quot((float)cab, Sf, rSf);
    const float p = v1 * v2, d = v3 - p, r = d * d;
    const double den = ((double)p * (1.0 - (double)v1)) * (1.0 - (double)v2);
    const double x = (double)r;
    double y = (1.0 / den) * (1.0 + seed_err), e = 0.0;
    for (int k = 0; k < 3; ++k) { e = fma(-den, y, 1.0); y = fma(y, e, y); }
    double q = x * y;
    q = fma(fma(-q, den, x), y, q);
    const long long mid = (long long)(d2b(q) & 0x1FFFFFFFull) - (1ll << 28);
    const int dz = den == 0.0, zero = ca == 0 || cb == 0;
    const int redo = !zero && !dz &&
                     (!(den > 0x1p-1000 && den < 0x1p1000) || (q != 0.0 && q < 0x1p-126) ||
                      (mid >= -64 && mid <= 64) || !(fabs(e) <= 0x1p-20));
    float f = dz ? b2f(r == 0.0f ? 0xFFC00000u
                                 : 0x7F800000u | ((uint32_t)(d2b(den) >> 32) & 0x80000000u))
                 : (float)q;
    if (f > b2f(0x3F800000u + 838u)) f = 123.456f;
    if (zero) f = 0.0f;
    if (redo) { ++fallbacks; f = ref_r2(cab, ca, cb, S); }
    return f;
}

int main(int argc, char **argv) {
    const long long N = argc > 1 ? atoll(argv[1]) : 1000000LL;
    long long bad = 0;
    for (long long i = 0; i < N; ++i) {
        const uint64_t k = rnd() % 4;
        const int S = k == 0 ? 2 + (int)(rnd() % 100)
                    : k == 1 ? 2 + (int)(rnd() % 20000) : 2 + (int)(rnd() % ((1u << 24) - 1));
        uint32_t ca = (uint32_t)(rnd() % (uint64_t)(S + 1)), cb = (uint32_t)(rnd() % (uint64_t)(S + 1));
        if (rnd() % 8 == 0) ca = (rnd() & 1) ? 1u : (uint32_t)S - 1;
        if (rnd() % 8 == 0) cb = (rnd() & 1) ? (uint32_t)S : 1u;
        if (rnd() % 64 == 0) ca = (uint32_t)S + (uint32_t)(rnd() % 50);   /* counts above S */
        const uint32_t mx = ca < cb ? ca : cb;
        uint32_t cab = (uint32_t)(rnd() % (uint64_t)(mx + 1));
        if (rnd() % 4 == 0) {   /* near independence: cab ~ ca*cb/S */
            long long c = llround((double)ca * cb / S) + (long long)(rnd() % 5) - 2;
            cab = (uint32_t)(c < 0 ? 0 : c > mx ? mx : c);
        }
        const double se = (urand() * 2 - 1) * 0x1p-8;
        const float a = ref_r2(cab, ca, cb, S), b = fast_r2(cab, ca, cb, S, se);
        if (f2b(a) != f2b(b)) {
            if (bad < 5)
                printf("mismatch S=%d cA=%u cB=%u cAB=%u ref=%.9g fast=%.9g\n", S, ca, cb, cab, a, b);
            ++bad;
        }
    }
    printf("pairs %lld mismatches %lld fallbacks %lld\n", N, bad, fallbacks);
    return bad != 0;
}
