/*
 * ref_harness.c -- entry points into the qLD reference's own compiled code.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
 * the reference's unmodified sources (src/correlator/src/gemm_cpu.c,
 * correlate_IO.c, fast_print.c, read_file.c) into oracle/_ref/libqldref.so.
 * Tests use it to pin the C restatement in qld_oracle.c, and bench.py's
 * reference arm times it as the reference CPU path.  The shipped library
 * never links it.
 *
 * Entry points:
 *   ref_counts_gemm    mlt() + gemm() exactly as correlate() calls them when
 *                      -blis is off (gemm_cpu.c:485, :535-546): full m x n
 *                      column-major uint64 counts.
 *   ref_ld_score       get_pairwise_ld_score() (gemm_cpu.c:343-404) on a slice
 *                      of B rows [i0, i1), so several threads can share a task.
 *   ref_write_report   writeResultsHeader() + writeResults()
 *                      (correlate_IO.c:378-429) into a file.
 *   ref_correlate      the whole per-task correlate() (gemm_cpu.c:420-623):
 *                      counts, epilogue and report, as qLD-compute runs it.
 */
#include <omp.h>

#include "correlate_IO.h"
#include "gemm_cpu.h"
#include "read_file.h"

void get_pairwise_ld_score(unsigned int *tableA_bitcount,
                           unsigned int *tableB_bitcount, inputDataType_x64 *C,
                           int tableAsize, int tableBsize, int snp_size,
                           ResultDataType **results);
void gemm(unsigned int m, unsigned int n, unsigned int k,
          inputDataType_x64 alphap, inputDataType_x64 *A, unsigned int lda,
          inputDataType_x64 *B, unsigned int ldb, inputDataType_x64 *C,
          unsigned int ldc, void *Ac_pack_v, void *Bc_pack_v);
void mlt(unsigned int m, unsigned int k, inputDataType_x64 *A,
         inputDataType_x64 *tableA);

#define REF_EXPORT __attribute__((visibility("default")))

REF_EXPORT int ref_counts_gemm(int m, int n, int K, const uint64_t *A,
                               const uint64_t *B, uint64_t *C)
{
    void *ac = NULL, *bc = NULL, *at = NULL;
    if (posix_memalign(&ac, 4096, 12 * BLOCK_MC * BLOCK_KC * sizeof(uint64_t)) ||
        posix_memalign(&bc, 4096, BLOCK_KC * BLOCK_NC * sizeof(uint64_t)) ||
        posix_memalign(&at, 4096, (size_t)m * K * sizeof(uint64_t) + 64))
        return -1;
    memset(C, 0, (size_t)m * n * sizeof(uint64_t));
    mlt((unsigned)m, (unsigned)K, (inputDataType_x64 *)at, (inputDataType_x64 *)A);
    gemm((unsigned)m, (unsigned)n, (unsigned)K, 1, (inputDataType_x64 *)at,
         (unsigned)m, (inputDataType_x64 *)B, (unsigned)K, C, (unsigned)m, ac, bc);
    free(ac);
    free(bc);
    free(at);
    return 0;
}

/* results (n x m, B-major) rows [i0, i1) from column-major counts C. */
REF_EXPORT void ref_ld_score(const uint32_t *bcA, const uint32_t *bcB,
                             const uint64_t *C, int m, int i0, int i1, int S,
                             float *results)
{
    float *slice = results + (size_t)i0 * m;
    get_pairwise_ld_score((unsigned int *)bcA, (unsigned int *)bcB + i0,
                          (inputDataType_x64 *)C + (size_t)i0 * m, m, i1 - i0, S,
                          &slice);
}

/* ref_ld_score over all n rows, split across nthreads OpenMP threads. */
REF_EXPORT void ref_ld_score_mt(const uint32_t *bcA, const uint32_t *bcB,
                                const uint64_t *C, int m, int n, int S,
                                float *results, int nthreads)
{
    if (nthreads < 1)
        nthreads = 1;
    int chunk = (n + nthreads * 4 - 1) / (nthreads * 4);
    if (chunk < 1)
        chunk = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int i0 = 0; i0 < n; i0 += chunk) {
        int i1 = i0 + chunk < n ? i0 + chunk : n;
        ref_ld_score(bcA, bcB, C, m, i0, i1, S, results);
    }
}

REF_EXPORT int ref_write_report(const char *path, const uint32_t *posA,
                                char **idA, const uint32_t *bcA, int m,
                                const uint32_t *posB, char **idB,
                                const uint32_t *bcB, int n, int S,
                                const float *results, float r2limit,
                                int posWset2)
{
    FILE *fp = fopen(path, "wb");
    if (!fp)
        return -1;
    writeResultsHeader(fp);
    writeResults(fp, (unsigned int *)posA, idA, (unsigned int *)bcA, m,
                 (unsigned int *)posB, idB, (unsigned int *)bcB, n, S,
                 (ResultDataType *)results, r2limit, posWset2);
    fclose(fp);
    return 0;
}

REF_EXPORT int ref_correlate(const char *out_path, const char *log_path,
                             const uint64_t *A, const uint32_t *posA, char **idA,
                             const uint32_t *bcA, int m, const uint64_t *B,
                             const uint32_t *posB, char **idB,
                             const uint32_t *bcB, int n, int K, int S,
                             int posWset2, float r2limit)
{
    threadData_t td;
    memset(&td, 0, sizeof td);
    td.threadTOTAL = 1;
    td.r2limit = r2limit;
    td.ploidy = 1;
    td.mdf = 1;
    td.threadLog = fopen(log_path, "w");
    FILE *fp = fopen(out_path, "wb");
    if (!fp || !td.threadLog)
        return -1;
    correlate(&td, fp, (inputDataType_x64 *)A, (unsigned int *)posA, idA,
              (unsigned int *)bcA, m, (inputDataType_x64 *)B,
              (unsigned int *)posB, idB, (unsigned int *)bcB, n, K, S, posWset2);
    fclose(fp);
    fclose(td.threadLog);
    return 0;
}
