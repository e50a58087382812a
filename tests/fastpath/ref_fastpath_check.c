/* CPU check of the branch-free reference-mode r^2 of the GPU epilogue
 * (qld_b200/csrc/epilogue.cuh: ref_factors, r2_reference_ff) against the
 * reference's operation sequence (qLD src/correlator/src/gemm_cpu.c:357-389),
 * bit for bit, over random pairs: small and large sample counts, fixed and
 * monomorphic SNPs, near-independence counts, bit counts above S.  The same
 * steps in C: per-row factors v = c/S, 1/(v(1-v)) as a float pair and 1/v;
 * the Markstein-corrected FP32 quotient cab/S; the FMA TwoProduct error of
 * p12; the quotient as a float pair; the rounding test and its fallback
 * (the fixed-SNP shortcut, else the literal sequence).  Build with -ffp-contract=off so the reference
 * sequence is not fused (fmaf() is an explicit FMA either way).
 *   usage: ref_fastpath_check N_PAIRS      exit 0 iff every pair matches */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t s_rng = 0x9E3779B97F4A7C15ull;
static uint64_t rnd(void) { s_rng ^= s_rng << 13; s_rng ^= s_rng >> 7; s_rng ^= s_rng << 17; return s_rng; }
static uint32_t f2b(float f) { uint32_t b; memcpy(&b, &f, 4); return b; }
static float b2f(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }

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
typedef struct { float v, hi, lo, iv; } Fac;
static Fac fac(uint32_t c, int S) {
    Fac f = {0, 0, 0, 0};
    if (c == 0) return f;
    float v = (float)c / (float)S;
    f.v = v;
    if (!(v < 1.0f)) { f.hi = NAN; f.iv = 1.0f; return f; }
    double om = 1.0 - (double)v;
    double i = 1.0 / ((double)v * om);
    f.hi = (float)i; f.lo = (float)(i - (double)f.hi); f.iv = 1.0f / v;
    return f;
}
static long long fallbacks = 0, fb_amb = 0, fb_tiny = 0, fb_spec = 0;

static float ff_r2(uint32_t cab, uint32_t ca, uint32_t cb, int S) {
    Fac A = fac(ca, S), B = fac(cb, S);
    const float Sf = (float)S, rSf = 1.0f / Sf;
    float cf = (float)cab;
    float q0 = cf * rSf; float v3 = fmaf(fmaf(-q0, Sf, cf), rSf, q0);
    float p12 = A.v * B.v; float e = fmaf(A.v, B.v, -p12);
    float d = v3 - p12; float x = d * d;
    float Ph = A.hi * B.hi; float Pl = fmaf(A.hi, B.hi, -Ph); Pl = fmaf(A.hi, B.lo, Pl); Pl = fmaf(A.lo, B.hi, Pl);
    float t = e * (A.iv * B.iv);
    float qh = x * Ph; float ql = fmaf(x, Ph, -qh); ql = fmaf(x, Pl, ql); ql = fmaf(qh, t, ql);
    float u = fmaf(qh, 0x1p-40f, ql), w = fmaf(qh, -0x1p-40f, ql);
    float rh = qh + u, rl = qh + w;
    uint32_t xb = f2b(x);
    int tiny = (xb - 1u) < (f2b(0x1p-100f) - 1u);
    int redo = (rh != rl) || tiny;
    float r = rh;
    if (r > b2f(0x3F800000u + 838u)) r = 123.456f;
    if (redo) {
        if (!(A.v > 0 && A.v < 1 && B.v > 0 && B.v < 1)) ++fb_spec; else if (tiny) ++fb_tiny; else ++fb_amb;
        ++fallbacks;
        /* the device's r2_flagged (and chunk_ref's pass over fixed A rows): zero rule,
         * fixed SNP (v = 1: den = +0) from the fast path's quotient v3, else the sequence */
        if (A.v == 0.0f || B.v == 0.0f) r = 0.0f;
        else if (A.v <= 1.0f && B.v <= 1.0f && (A.v == 1.0f || B.v == 1.0f)) {
            volatile float q = v3, p = A.v * B.v;
            volatile float dd = q - p, xx = dd * dd;
            r = xx == 0.0f ? b2f(0xFFC00000u) : 123.456f;
        } else r = ref_r2(cab, ca, cb, S);
    }
    return r;
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
        if (rnd() % 64 == 0) ca = (uint32_t)S + (uint32_t)(rnd() % 50);
        const uint32_t mx = ca < cb ? ca : cb;
        uint32_t cab = (uint32_t)(rnd() % (uint64_t)(mx + 1));
        if (rnd() % 4 == 0) {
            long long c = llround((double)ca * cb / S) + (long long)(rnd() % 5) - 2;
            cab = (uint32_t)(c < 0 ? 0 : c > mx ? mx : c);
        }
        const float a = ref_r2(cab, ca, cb, S), b = ff_r2(cab, ca, cb, S);
        if (f2b(a) != f2b(b)) {
            if (bad < 5) printf("mismatch S=%d cA=%u cB=%u cAB=%u ref=%.9g fast=%.9g\n", S, ca, cb, cab, a, b);
            ++bad;
        }
    }
    printf("pairs %lld mismatches %lld fallbacks %lld (special %lld tiny %lld ambiguous %lld)\n", N, bad, fallbacks, fb_spec, fb_tiny, fb_amb);
    return bad != 0;
}
