/*
 * ref_blis.c -- the reference's stock fast CPU path, timed.
 *
 * CPU-BASELINE AND TEST INFRASTRUCTURE ONLY.  oracle/Makefile links this file with
 * the reference's unmodified gemm_cpu.c compiled as its `cblas_cpu_syrk`
 * target compiles it (-DCBLAS_USE -DSYRK, src/correlator/Makefile:31-39) and
 * with BLIS 0.1.8 configured for `binary_gemm` (the qLD-vendored BLIS, its
 * framework plus the bin_gemm_2x2 AND+POPCNT micro-kernel), into
 * oracle/_ref/libqldref_blis.so.  bench.py's reference arm times it.
 *
 *   refb_counts_ld   what correlate() runs between its "GEMM" and "LD"
 *                    timers with -blis (gemm_cpu.c:517-563): blis_gemm()
 *                    -- cblas_dsyrk (lower) for a single region, cblas_dgemm
 *                    for two -- then get_pairwise_ld_score() on one thread.
 *                    C and results are zeroed first, outside the timers, as
 *                    correlate() does at :477-483.  BLIS threads follow
 *                    BLIS_JC_NT / BLIS_IC_NT / ... read from the environment
 *                    at each call.
 */
#include <fcntl.h>
#include <stdio.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "gemm_cpu.h"

void get_pairwise_ld_score(unsigned int *tableA_bitcount,
                           unsigned int *tableB_bitcount, inputDataType_x64 *C,
                           int tableAsize, int tableBsize, int snp_size,
                           ResultDataType **results);

#define REF_EXPORT __attribute__((visibility("default")))

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* counts (column-major m x n uint64) and results (n x m float, B-major) of
 * one task; B == A and posWset == 0 for a single region.  Seconds spent in
 * the counts and in the epilogue go to t_gemm / t_ld. */
REF_EXPORT int refb_counts_ld(int m, int n, int K, const uint64_t *A, const uint64_t *B,
                              const uint32_t *bcA, const uint32_t *bcB, int S, int posWset,
                              uint64_t *C, float *results, double *t_gemm, double *t_ld)
{
    memset(C, 0, (size_t)m * n * sizeof(uint64_t));
    memset(results, 0, (size_t)m * n * sizeof(float));
    /* blis_gemm() prints a line per call on stdout; keep it off the
     * caller's stdout (outside the timers). */
    fflush(stdout);
    int saved = dup(1), nul = open("/dev/null", O_WRONLY);
    if (saved >= 0 && nul >= 0)
        dup2(nul, 1);
    double t0 = now_s();
    blis_gemm((unsigned)m, (unsigned)n, (unsigned)K, 1, (inputDataType_x64 *)A,
              (inputDataType_x64 *)B, (inputDataType_x64 *)C, posWset);
    double t1 = now_s();
    fflush(stdout);
    if (saved >= 0 && nul >= 0)
        dup2(saved, 1);
    if (saved >= 0)
        close(saved);
    if (nul >= 0)
        close(nul);
    double t2 = now_s();
    get_pairwise_ld_score((unsigned int *)bcA, (unsigned int *)bcB, (inputDataType_x64 *)C, m, n,
                          S, &results);
    double t3 = now_s();
    *t_gemm = t1 - t0;
    *t_ld = t3 - t2;
    return 0;
}
