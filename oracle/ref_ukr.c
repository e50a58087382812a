/*
 * ref_ukr.c -- a BLIS-style blocked loop around the reference's own binary
 * GEMM micro-kernel bin_gemm_2x2 (blis/config/binary_gemm/kernels/3/bin_gemm.c:4-141).
 *
 * TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.  qLD's fast CPU path is BLIS 0.1.8's
 * dsyrk/dgemm with this micro-kernel plugged in (gemm_cpu.c:195-237), which
 * oracle/Makefile builds from BLIS's sources (ref_blis.c times it).  This
 * file is the stand-in bench.py falls back to, and says so, where that BLIS
 * build is absent: BLIS's blocking and packing around the reference kernel,
 * with the block sizes of the binary_gemm configuration
 * (blis/config/binary_gemm/bli_kernel.h:84-89: MC=72, KC=256, NC=4080,
 * MR=NR=2) and OpenMP threads over column blocks, as BLIS_JC_NT would split
 * them.
 *
 * Packing follows what the micro-kernel reads: an MR x KC micro-panel of A
 * stored k-major (a[ir + l*MR]), a KC x NR micro-panel of B stored the same
 * way (b[jr + l*NR]); C is column-major m x n uint64, as in blis_gemm().
 * Edge micro-tiles are padded with zero rows and go through a 2x2 scratch.
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "blis.h"

void bin_gemm_2x2(dim_t k, double *restrict alpha, double *restrict a,
                  double *restrict b, double *restrict beta, double *restrict c,
                  inc_t rs_c, inc_t cs_c, auxinfo_t *data);

enum { U_MC = 72, U_KC = 256, U_NC = 4080, U_MR = 2, U_NR = 2, U_NB = 96 };

static void pack_panel(const uint64_t *X, int rows, int r0, int nr, int K,
                       int k0, int kc, uint64_t *dst)
{
    /* rows [r0, r0+nr) of row-major X (K words per row), k in [k0, k0+kc),
     * as a 2-wide micro-panel: dst[i + l*2]; missing rows are zero. */
    for (int l = 0; l < kc; l++)
        for (int i = 0; i < 2; i++) {
            int r = r0 + i;
            dst[i + l * 2] = (i < nr && r < rows) ? X[(size_t)r * K + k0 + l] : 0;
        }
}

__attribute__((visibility("default")))
int ref_counts_ukr(int m, int n, int K, const uint64_t *A, const uint64_t *B,
                   uint64_t *C, int lower_only, int nthreads)
{
    if (nthreads < 1)
        nthreads = 1;
    int nblk = (n + U_NB - 1) / U_NB;
    int err = 0;
#pragma omp parallel num_threads(nthreads)
    {
        void *apv = NULL, *bpv = NULL;
        if (posix_memalign(&apv, 64, sizeof(uint64_t) * (U_MC + 2) * U_KC))
            apv = NULL;
        if (posix_memalign(&bpv, 64, sizeof(uint64_t) * (U_NB + 2) * U_KC))
            bpv = NULL;
        uint64_t *ap = apv, *bp = bpv;
        if (!ap || !bp) {
#pragma omp atomic write
            err = -1;
        }
#pragma omp for schedule(dynamic, 1)
        for (int jb = 0; jb < nblk; jb++) {
            if (!ap || !bp)
                continue;
            int j0 = jb * U_NB;
            int nb = n - j0 < U_NB ? n - j0 : U_NB;
            int i_start = lower_only ? (j0 / U_MC) * U_MC : 0;
            for (int k0 = 0; k0 < K; k0 += U_KC) {
                int kc = K - k0 < U_KC ? K - k0 : U_KC;
                double alpha = 1.0, beta = (k0 == 0) ? 0.0 : 1.0;
                for (int jr = 0; jr < nb; jr += U_NR)
                    pack_panel(B, n, j0 + jr, nb - jr, K, k0, kc, bp + (size_t)jr * kc);
                for (int i0 = i_start; i0 < m; i0 += U_MC) {
                    int mb = m - i0 < U_MC ? m - i0 : U_MC;
                    for (int ir = 0; ir < mb; ir += U_MR)
                        pack_panel(A, m, i0 + ir, mb - ir, K, k0, kc, ap + (size_t)ir * kc);
                    for (int jr = 0; jr < nb; jr += U_NR) {
                        for (int ir = 0; ir < mb; ir += U_MR) {
                            int a = i0 + ir, b = j0 + jr;
                            if (lower_only && a + 1 < b)
                                continue; /* micro-tile wholly above the diagonal */
                            double tmp[4];
                            uint64_t *t = (uint64_t *)tmp;
                            int full = (ir + 2 <= mb) && (jr + 2 <= nb);
                            if (full) {
                                bin_gemm_2x2(kc, &alpha, (double *)(ap + (size_t)ir * kc),
                                             (double *)(bp + (size_t)jr * kc), &beta,
                                             (double *)(C + a + (size_t)b * m), 1, m, NULL);
                            } else {
                                double zero = 0.0;
                                bin_gemm_2x2(kc, &alpha, (double *)(ap + (size_t)ir * kc),
                                             (double *)(bp + (size_t)jr * kc), &zero,
                                             tmp, 1, 2, NULL);
                                for (int y = 0; y < 2 && jr + y < nb; y++)
                                    for (int x = 0; x < 2 && ir + x < mb; x++) {
                                        uint64_t *dst = C + (a + x) + (size_t)(b + y) * m;
                                        *dst = (beta == 0.0 ? 0 : *dst) + t[x + 2 * y];
                                    }
                            }
                        }
                    }
                }
            }
        }
        free(ap);
        free(bp);
    }
    if (lower_only) /* SYRK leaves the strict upper triangle at 0 */
        for (int b = 0; b < n; b++)
            for (int a = 0; a < b && a < m; a++)
                C[a + (size_t)b * m] = 0;
    return err;
}
