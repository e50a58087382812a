// qld_kernels.h -- host-side view of the counts kernels (internal to libqld_cuda).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "qld_cuda.h"
#include "qld_device.cuh"

namespace qld {

// Geometry a launcher needs from a kernel: output tile, and the TMA box
// (box_words words along K by box_rows rows) its tensor maps must use.
struct KernelShape {
    int bm, bn;       // A rows x B rows per output tile
    int box_words;    // K words per TMA box (one stage)
    int box_rows_a;   // rows per TMA box of the A map
    int box_rows_b;   // rows per TMA box of the B map
    int swizzle;      // TMA swizzle span in bytes (64 or 128)
};

extern const KernelShape kPopcShape;
extern const KernelShape kMmaShape;       // 128 x 256 tiles, overlapped epilogue
extern const KernelShape kMmaWideShape;   // 256 x 256 tiles

// Variant (a): tiles_b tile rows starting at p.tb0; p.nk = ceil(K / box_words).
cudaError_t launch_popc(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                        int tiles_b, int r2_mode, cudaStream_t st);

// Variant (b): p.nk unused (the kernel derives its stages from K).  Exact
// while K * 64 <= kMmaMaxSamples.
extern const int kMmaMaxSamples;
cudaError_t launch_mma(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                       int tiles_b, int r2_mode, cudaStream_t st);
cudaError_t launch_mma_wide(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                            int tiles_b, int r2_mode, cudaStream_t st);

// Variant (c): bits as E2M1 on tcgen05.mma.kind::mxf4 with F32 accumulators,
// 256 x 240 tiles.  Exact while K * 64 <= kMxf4MaxSamples.
extern const KernelShape kMxf4Shape;
extern const int kMxf4MaxSamples;
cudaError_t launch_mxf4(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                        int tiles_b, int r2_mode, cudaStream_t st);
// The same tiles computed by clusters of two CTAs (one per SM, 128 A rows and
// 120 B rows each), with the epilogue overlapping the next tile's MMAs.
extern const KernelShape kMxf4PairShape;
cudaError_t launch_mxf4_pair(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                             int tiles_b, int r2_mode, cudaStream_t st);

// One task of a batched launch: its tensor maps (kBatchShape boxes), sizes,
// output, and the number of work items (output tiles) of the tasks before it.
struct BatchJob {
    CUtensorMap tmA, tmB;
    const uint32_t *bcA, *bcB;
    float *r2;
    uint32_t *counts;
    long long ldr, ldc;
    long long item0;
    int m, n, K, S, symmetric;
    float threshold;           // with summary: the n_above threshold
    BatchSummary *summary;     // NULL: none
};

struct BatchParams {
    const BatchJob *jobs;
    int njobs;
    long long nitems;
    unsigned long long *queue;   // work-queue ticket counter, zero at launch
    unsigned *status;
    long long timeout_cycles;
};

extern const KernelShape kBatchShape;   // 256 x 240 tiles on SM pairs, the 4-bit path
extern const int kBatchMaxSamples;      // K * 64 limit of a batched task (2^24)

// Persistent batched launch over all items of bp.jobs (max_ctas > 0 caps the grid).
cudaError_t launch_batch(const BatchParams &bp, int r2_mode, int max_ctas, cudaStream_t st);

// COUNTSTATES (ld_states.cu): state value of every pair, one byte each at
// out[(b - out_row0) * lds + a]; single region: only a >= b.
struct StatesParams {
    int m, n, K, symmetric;
    int tb0;                  // first B tile of this launch
    uint8_t *out;
    long long lds;
    int out_row0;
    unsigned *status;
    long long timeout_cycles;
};
extern const KernelShape kStatesShape;
cudaError_t launch_states(const CUtensorMap &tmA, const CUtensorMap &tmB, const StatesParams &p,
                          int tiles_b, cudaStream_t st);

// VCF sites -> packed rows (vcf_pack.cu).  With rnd_off NULL the launch only
// counts: per site the random draws its unphased genotypes need
// (slash_count), its row length and count-stage errors.  Otherwise it packs,
// drawing site s's numbers from rnd[rnd_off[s]...].  Each CTA uses
// scratch_cap bytes of scratch (>= K * 64).
enum VcfError {
    QLD_VCF_OK = 0,
    QLD_VCF_EMPTY_GT = 1,     // the GT subfield is empty
    QLD_VCF_ALLELE = 2,       // an allele index past the REF/ALT states
    QLD_VCF_ALLELES = 3,      // more than three alleles in a genotype
    QLD_VCF_SAMPLES = 4,      // more sample fields than header samples
    QLD_VCF_PLOIDY = 5,       // a genotype bigger than the ploidy
    QLD_VCF_SHORT_GT = 6,     // fewer alleles than the genotype's separators say
    QLD_VCF_NO_SAMPLES = 7,   // no alleles at all
    QLD_VCF_STATE_CHAR = 8,   // a REF/ALT character qLD cannot map (lower case, '.')
};
cudaError_t launch_vcf_sites(const char *text, const qld_vcf_site *sites, int nsites,
                             const uint8_t *valid, int nsamples, int ploidy, int K,
                             const unsigned *rnd, const long long *rnd_off,
                             long long *slash_count, char *scratch, int scratch_cap, int ctas,
                             uint64_t *words, uint32_t *bc, int *snip_len, uint8_t *keep,
                             int *err, cudaStream_t st);

// Report filter over `rows` r^2 rows (ldr >= m rounded up to 128 floats,
// 16-byte aligned rows): mask (rows x W words, W = ceil(m / 32)), per-row
// counts, offsets (rows + 1) and the kept values (hits.cu).  Row r is B row
// row0 + r; with `triangle` only columns j > row0 + r are kept.
cudaError_t launch_hits(const float *r2, long long ldr, int rows, int m, int row0, int triangle,
                        float r2limit, uint32_t *mask, int W, long long *cnt, long long *off,
                        float *val, cudaStream_t st);

// Rows of K words back to back (a staging copy of a host table) -> rows of
// ldd >= K words, words past K zeroed (rows.cu).
cudaError_t launch_pad_rows(uint64_t *dst, long long ldd, const uint64_t *src, int K,
                            long long rows, cudaStream_t st);

}  // namespace qld
