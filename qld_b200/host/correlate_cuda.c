/*
 * correlate_cuda.c -- qLD-compute's -cuda mode: correlate() on a B200.
 *
 * Drop-in source for qLD's src/correlator/src/ (it includes the correlator's
 * own headers, found through the Makefile's -Iinclude/).  correlate_cuda()
 * has exactly the argument list of correlate() (src/correlator/include/
 * gemm_cpu.h:24-38) and does what correlate() does (gemm_cpu.c:420-623) with
 * the counts and the r^2 epilogue (gemm_cpu.c:517-563) replaced by one call
 * to libqld_cuda (include/qld_cuda.h); the report is written by the
 * reference's own writeResultsHeader()/writeResults() (correlate_IO.c:378-429),
 * so the output file layout is unchanged.
 *
 * Context: one libqld_cuda context per worker thread, created on the thread's
 * first task (the role gpu_init() plays for -gpu, correlate_our_kernel.c:593-596)
 * on device QLD_CUDA_DEVICE (default 0) and released by qld_cuda_thread_release().
 * r^2 mode: reference semantics (bit-identical results[], byte-identical
 * report) unless QLD_R2=exact selects the exact-D FP64-evaluated r^2.
 * The pinned results[] buffer (correlate()'s m x n floats, gemm_cpu.c:467)
 * is kept per thread and only grows, so an -inputList run pins host memory
 * once instead of once per task (a 29,817-SNP region needs 3.6 GB).
 * Errors keep qLD-compute's behaviour: a message on stderr and exit(1).
 *
 * Single region: the symmetric (lower-triangle) computation is used only when
 * table B is table A.  For split-file input lists qLD sets posWset2 = 0 with
 * a different table B (load_balancer.c:262-268); the full A x B counts are
 * computed then, as the reference's fallback gemm() does, and writeResults()
 * prints the triangle as before.
 */
#include <stdlib.h>

#include "correlate_IO.h"
#include "gemm_cpu.h"
#include "header.h"
#include "qld_cuda.h"
#include "read_file.h"

static __thread qld_ctx *tls_ctx = NULL;
static __thread float *tls_results = NULL;   /* pinned, tls_cap floats */
static __thread size_t tls_cap = 0;

static void cuda_fail(const char *what, int rc)
{
    fprintf(stderr, "qLD-compute: -cuda: %s failed (%d): %s\n", what, rc,
            tls_ctx ? qld_cuda_last_error(tls_ctx) : "no context");
    exit(1);
}

static qld_ctx *thread_ctx(void)
{
    if (!tls_ctx) {
        const char *d = getenv("QLD_CUDA_DEVICE");
        int rc = qld_cuda_init(d ? atoi(d) : 0, &tls_ctx);
        if (rc != QLD_OK)
            cuda_fail("qld_cuda_init", rc);
        const char *mode = getenv("QLD_R2");
        rc = qld_cuda_set_option(tls_ctx, QLD_OPT_R2_MODE,
                                 (mode && !strcmp(mode, "exact")) ? QLD_R2_EXACT
                                                                  : QLD_R2_REFERENCE);
        if (rc != QLD_OK)
            cuda_fail("qld_cuda_set_option", rc);
    }
    return tls_ctx;
}

/* The thread's pinned results[] buffer, grown to at least `cells` floats. */
static float *thread_results(qld_ctx *ctx, size_t cells)
{
    if (cells > tls_cap) {
        if (tls_results)
            qld_cuda_host_free(ctx, tls_results);
        tls_results = NULL;
        tls_cap = 0;
        int rc = qld_cuda_host_alloc(ctx, cells * sizeof(float), (void **)&tls_results);
        if (rc != QLD_OK)
            cuda_fail("qld_cuda_host_alloc", rc);
        tls_cap = cells;
    }
    return tls_results;
}

void qld_cuda_thread_release(void)
{
    if (tls_ctx) {
        if (tls_results)
            qld_cuda_host_free(tls_ctx, tls_results);
        tls_results = NULL;
        tls_cap = 0;
        qld_cuda_release(tls_ctx);
        tls_ctx = NULL;
    }
}

void correlate_cuda(threadData_t *threadData,
                    outFileType fpOut,
                    inputDataType_x64 *tableA,
                    unsigned int *tableA_posIndex,
                    char **tableA_IDindex,
                    unsigned int *tableA_bitcount,
                    int tableAsize,
                    inputDataType_x64 *tableB,
                    unsigned int *tableB_posIndex,
                    char **tableB_IDindex,
                    unsigned int *tableB_bitcount,
                    int tableBsize,
                    int compressed_snp_size,
                    int snp_size,
                    int posWset2)
{
    double t0 = gettime();
    qld_ctx *ctx = thread_ctx();
    int m = tableAsize, n = tableBsize;
    int symmetric = (posWset2 == 0 && tableA == tableB && m == n);
    size_t cells = (size_t)m * (size_t)n;
    float *results = thread_results(ctx, cells ? cells : 1);

    writeResultsHeader(fpOut);
    double t1 = gettime();
    int rc = qld_cuda_ld(ctx, tableA, tableA_bitcount, m, tableB, tableB_bitcount, n,
                         compressed_snp_size, snp_size, symmetric, results, NULL);
    if (rc != QLD_OK)
        cuda_fail("qld_cuda_ld", rc);
    double t2 = gettime();

    writeResults(fpOut, tableA_posIndex, tableA_IDindex, tableA_bitcount, m,
                 tableB_posIndex, tableB_IDindex, tableB_bitcount, n, snp_size,
                 results, threadData[0].r2limit, posWset2);
    double t3 = gettime();

#if defined(VERBOSE) || defined(BENCHMARK)
    threadData[0].threadStats.init_time += t1 - t0;
    threadData[0].threadStats.gemm_time += t2 - t1;
    threadData[0].threadStats.write_time += t3 - t2;
    fprintf(threadData[0].threadLog, "[T] Init times: %f\n", t1 - t0);
    fprintf(threadData[0].threadLog, "[T] GEMM+LD times (cuda): %f\n", t2 - t1);
    fprintf(threadData[0].threadLog, "[T] Write times: %f\n\n", t3 - t2);
#else
    (void)t0; (void)t1; (void)t2; (void)t3;
#endif
}
