/*
 * qld_cuda.h -- C ABI of libqld_cuda, the sm_100a (B200) LD hot path of
 * qLD-compute: pairwise AND+popcount counts over packed 64-bit MDF rows and
 * the fused r^2 epilogue.
 *
 * Plain C types only (no CUDA or torch types): a C caller such as
 * qLD-compute's per-task driver links it directly; other hosts bind it
 * through their FFI.  Every function returns QLD_OK (0) or a negative
 * QLD_ERR_* code and never exits the process; qld_cuda_last_error() gives the
 * message of the last failure on a context.
 *
 * Data layout (as qLD's table_x64, src/correlator/include/correlate_MEM.h:66-75):
 *   A, B     row-major SNP tables, K uint64 words per row, MSB-first packing
 *            (sample s is bit 63 - s%64 of word s/64), zero tail bits.
 *   bcA, bcB per-row popcounts (the MDF BC field, BCtable).
 *   r2_out   n x m float, B-major: r2_out[i*m + j] is the r^2 of B row i and
 *            A row j -- the reference's results[] (gemm_cpu.c:357-388).
 *   counts   n x m uint32 with the same indexing, i.e. the reference's
 *            column-major m x n C matrix (gemm_cpu.c:203-236) narrowed to 32 bit.
 *   symmetric  single-region task (the reference's posWset2 == 0): B is A and
 *            only entries with j >= i (A index >= B index: the lower triangle of
 *            C including its diagonal, what cblas_dsyrk(CblasLower) fills) are
 *            defined on return; the entries with j < i are unspecified (the
 *            reference leaves values there that its writer never reads).
 *
 * r^2 modes (per entry, cA = bcA[j], cB = bcB[i], c = count, S = snp_size):
 *   QLD_R2_EXACT      r^2 = D^2 / (cA(S-cA) cB(S-cB)) with the exact integer
 *                     D = S*c - cA*cB; relative error <= 1e-6 against an
 *                     FP64 oracle.  The popcount and int8 kernels evaluate in
 *                     FP64 and round once (<= 2^-24); the 4-bit kernels in
 *                     FP32 from their exact F32 counts, D to 3 * 2^-24 and
 *                     r^2 to 11 * 2^-24 (6.6e-7).  Zeros, NaN and 123.456
 *                     are identical in every kernel.
 *   QLD_R2_REFERENCE  bit-identical to get_pairwise_ld_score()
 *                     (gemm_cpu.c:343-404): FP32 frequencies, FP32 numerator,
 *                     FP64 denominator, no fused multiply-add.
 *   Both: r^2 = 0 when cA == 0 or cB == 0; r^2 > 1.0001 becomes 123.456;
 *   0/0 (an all-ones SNP) stays NaN.
 */
#ifndef QLD_CUDA_H
#define QLD_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QLD_CUDA_ABI_VERSION 1

/* status codes */
#define QLD_OK               0
#define QLD_ERR_INVALID     -1  /* bad argument                                  */
#define QLD_ERR_CUDA        -2  /* a CUDA runtime/driver call failed             */
#define QLD_ERR_NOMEM       -3  /* device or pinned host allocation failed       */
#define QLD_ERR_NODEVICE    -4  /* no usable sm_100 device                       */
#define QLD_ERR_TIMEOUT     -5  /* a kernel's bounded wait gave up               */
#define QLD_ERR_BUSY        -6  /* admission refused (serving)                   */
#define QLD_ERR_UNSUPPORTED -7  /* shape/option not supported by this kernel     */
#define QLD_ERR_TOO_LARGE   -8  /* task does not fit qld_cuda_ld_noalloc's scratch */

/* r^2 evaluation modes */
#define QLD_R2_EXACT      0
#define QLD_R2_REFERENCE  1

/* counts-kernel variants */
#define QLD_KERNEL_AUTO   0  /* per-shape choice                                 */
#define QLD_KERNEL_POPC   1  /* LOP3 + POPC on the CUDA cores                     */
#define QLD_KERNEL_MMA    2  /* bit -> int8 unpack + tcgen05 i8 MMA (TMEM)        */
#define QLD_KERNEL_FP4    3  /* bit -> E2M1 unpack + tcgen05 block-scaled MXF4 MMA */

/* qld_cuda_set_option() keys */
#define QLD_OPT_KERNEL    1  /* QLD_KERNEL_*                                      */
#define QLD_OPT_R2_MODE   2  /* QLD_R2_*                                          */
#define QLD_OPT_PROFILE   3  /* 1: time every counts-kernel launch with events    */
#define QLD_OPT_BAND_ROWS 4  /* B rows per streamed output band (host-buffer calls);
                                rounded down to whole tile rows of the kernel */
#define QLD_OPT_MMA_TILE  5  /* QLD_KERNEL_MMA output tile rows: 128, 256, 0 = per shape */
#define QLD_OPT_SM_PAIR   6  /* QLD_KERNEL_FP4 SMs per output tile: 1, 2 (a cluster of two
                                CTAs, tcgen05 cta_group::2), 0 = automatic (the tuned
                                choice for the task's class, else 2) */
#define QLD_OPT_WAIT_CYCLES 7 /* budget of every bounded wait inside the kernels' pipelines,
                                in SM clock cycles (0 = the default 4e9, ~2 s; the environment
                                variable QLD_TIMEOUT_CYCLES sets the initial value).  A wait
                                that runs out records the cause and the kernel ends early:
                                the call returns QLD_ERR_TIMEOUT and the context stays usable.
                                Copies and MMAs in flight are always drained first. */
#define QLD_OPT_MEM_CAP   8  /* cap, in bytes, on the device buffers the context allocates
                                for its calls (0 = no cap).  A call that would grow them past
                                it returns QLD_ERR_NOMEM before launching anything; the
                                context stays usable.  Buffers already held count toward the
                                cap and are kept (a lower cap applies as they grow). */

typedef struct qld_ctx qld_ctx;

/*
 * Context lifecycle.  Replaces gpu_init()/gpu_release() (qLD
 * src/correlator/include/gemm_gpu.h:52-54, called from
 * correlate_our_kernel.c:593-596,626-629).  One context per host thread;
 * a context is not re-entrant.
 */
int qld_cuda_init(int device, qld_ctx **ctx_out);
int qld_cuda_release(qld_ctx *ctx);
const char *qld_cuda_last_error(const qld_ctx *ctx);
int qld_cuda_set_option(qld_ctx *ctx, int option, long long value);

/*
 * One LD task from host memory: the counts + r^2 part of correlate()
 * (gemm_cpu.c:420-623: blis_gemm()/gemm() at :517-547 and
 * get_pairwise_ld_score() at :557-563), with qLD-compute's argument meaning:
 * m = tableAsize, n = tableBsize, K = compressed_snp_size, S = snp_size,
 * symmetric = (posWset2 == 0).  B/bcB are ignored when symmetric (n must
 * equal m).  counts_out may be NULL.  Host buffers may be pageable or pinned
 * (qld_cuda_host_alloc); pinned ones let the copies overlap the kernels.
 * Synchronous: returns when r2_out (and counts_out) hold the results.
 */
int qld_cuda_ld(qld_ctx *ctx,
                const uint64_t *A, const uint32_t *bcA, int m,
                const uint64_t *B, const uint32_t *bcB, int n,
                int K, int S, int symmetric,
                float *r2_out, uint32_t *counts_out);

/*
 * The same task on device-resident buffers, enqueued on `stream`
 * (a cudaStream_t; NULL = the context's own stream, which is non-blocking:
 * pass cudaStreamLegacy, or the stream that writes the inputs, to order the
 * call after work on the legacy default stream), asynchronous.
 *   lda/ldb   words between consecutive rows in device memory (>= K, even;
 *             row starts 16-byte aligned).  Words past K are never read.
 *   ldr/ldc   elements between consecutive B rows of r2 / counts (>= m).
 * Call qld_cuda_sync() to wait and collect the kernel status.
 */
typedef struct qld_ld_args {
    const uint64_t *A; const uint32_t *bcA; int m; long long lda;
    const uint64_t *B; const uint32_t *bcB; int n; long long ldb;
    int K; int S; int symmetric;
    float *r2; long long ldr;
    uint32_t *counts; long long ldc;
} qld_ld_args;

int qld_cuda_ld_device(qld_ctx *ctx, const qld_ld_args *args, void *stream);
int qld_cuda_sync(qld_ctx *ctx, void *stream);

/*
 * One task split over several GPUs (one context per GPU, each holding the
 * whole tables): part `part` of `nparts` computes the B rows
 * [*row0, *row1) -- consecutive whole tile rows of the kernel the context
 * chooses, with (nearly) equal numbers of output tiles, i.e. equal bit-ops --
 * into args->r2 / args->counts, whose row 0 is B row *row0 (so they need
 * *row1 - *row0 rows).  No exchange between the parts: each GPU keeps its
 * rows.  Parts past a task's last tile row are empty (*row0 == *row1).
 * qld_cuda_split_rows gives the same ranges without a context or a GPU, for
 * kernel QLD_KERNEL_POPC / _MMA / _FP4 (AUTO: the built-in rule).
 * No counterpart in the reference (its tasks are split by the user's window
 * lists, load_balancer.c / utilities/split_region, one CPU thread each).
 */
int qld_cuda_ld_device_part(qld_ctx *ctx, const qld_ld_args *args, int part, int nparts,
                            int *row0, int *row1, void *stream);
int qld_cuda_split_rows(int m, int n, int K, int symmetric, int kernel, int part, int nparts,
                        int *row0, int *row1);

/*
 * The report's pairs only, filtered on the GPU.  Computes the task as
 * qld_cuda_ld() does, one block of QLD_OPT_BAND_ROWS B rows at a time, and
 * keeps the pairs qLD's writeResults() prints (src/correlator/src/
 * correlate_IO.c:403-409): r2limit <= r^2 < 100, and with `triangle` only
 * j > i (qLD's posWset2 == 0; implied by `symmetric`).  Each block crosses
 * PCIe as a bit mask (m/8 bytes per row) plus the passing values, and is
 * handed to `fn` on the calling thread while the GPU computes the next
 * block.  The block's arrays are valid during the call only.  `fn` returns 0
 * to go on; any other value stops the task and is returned.
 */
typedef struct qld_hits_block {
    int row0, rows;            /* B rows [row0, row0 + rows) */
    int m;                     /* columns: A rows */
    int words;                 /* mask words per row: ceil(m / 32) */
    const uint32_t *mask;      /* rows x words: bit (j & 31) of word j >> 5 set <=> (row, j) kept */
    const long long *row_off;  /* rows + 1 offsets into val, row_off[0] == 0 */
    const float *val;          /* the kept r^2 of each row, in column order */
} qld_hits_block;
typedef int (*qld_hits_fn)(void *user, const qld_hits_block *block);
int qld_cuda_ld_hits(qld_ctx *ctx, const uint64_t *A, const uint32_t *bcA, int m,
                     const uint64_t *B, const uint32_t *bcB, int n, int K, int S, int symmetric,
                     int triangle, float r2limit, qld_hits_fn fn, void *user);

/*
 * COUNTSTATES: qLD-compute's -DCOUNTSTATES build replaces the r^2 task by
 * countStates_mode() (src/correlator/src/correlate_IO.c:472-516).  For every
 * pair a state value: st = 0, then per 64-bit word st = popcount(st | S),
 * S = the joint states (A bit, B bit) present among the word's 64 bit pairs
 * (bit 2*a + b); the zero tail bits of the last word count as state (0,0).
 * states_out[i*m + j] (B-major, one byte) for B row i and A row j; with
 * `symmetric` (B is A) only entries j >= i are defined.  Host-buffer and
 * device forms as qld_cuda_ld / qld_cuda_ld_device (lds >= m bytes between
 * B rows).
 */
int qld_cuda_count_states(qld_ctx *ctx, const uint64_t *A, int m, const uint64_t *B, int n,
                          int K, int symmetric, uint8_t *states_out);
int qld_cuda_count_states_device(qld_ctx *ctx, const uint64_t *A, int m, long long lda,
                                 const uint64_t *B, int n, long long ldb, int K, int symmetric,
                                 uint8_t *states, long long lds, void *stream);

/*
 * VCF -> MDF packing on the GPU: the per-sample half of qLD-parse-2MDF
 * (src/mdf_extension/src/process_data.c:152-328, snip_processing.c).  Each
 * site is one VCF data line that passed its fixed-field checks: the bytes of
 * its sample fields in `text` (separated by spaces/tabs), the index of GT in
 * FORMAT and the REF/ALT state characters.  Per site: the valid samples'
 * alleles (getGTfield/getGTdata: digits -> states, '.' -> 'N', unphased
 * '/' groups shuffled with rand()), qLD's polymorphism test and the packed
 * row -- K words MSB-first, bit 1 for a base other than the site's first
 * base -- with its BC.  `rng` is called once per random draw, in qLD's order
 * (libc rand() reproduces qLD's shuffles); it may be NULL when no genotype
 * is unphased.  Outputs per site: words (nsites x K), bc, snip_len (alleles
 * in the row), keep (1: the row goes to the MDF).  A data error returns
 * QLD_ERR_INVALID with the first failing site in *err_site (else -1).
 */
typedef struct qld_vcf_site {
    long long off;      /* first byte of the line's sample fields in text */
    int len;            /* bytes from there to the end of the line */
    int gt_pos;         /* index of GT among the FORMAT subfields */
    int n_states;       /* REF + ALT states */
    char states[4];     /* REF, then ALT ('.' replaced by REF) */
} qld_vcf_site;
typedef unsigned (*qld_rand_fn)(void *user);
int qld_cuda_vcf_pack(qld_ctx *ctx, const char *text, size_t text_bytes,
                      const qld_vcf_site *sites, int nsites, const uint8_t *valid, int nsamples,
                      int ploidy, int K, qld_rand_fn rng, void *rng_user, uint64_t *words,
                      uint32_t *bc, int *snip_len, uint8_t *keep, int *err_site);

/*
 * Windowed (band) LD over one region: r^2 only for SNP pairs (i, j) with
 * 1 <= j - i <= band.  Output is the m x band array r2_band[i*band + d] =
 * r^2(SNP i, SNP i+1+d) (entries with i+1+d >= m are unspecified); counts_band
 * (optional) likewise.  The host-buffer form streams: the table goes to the
 * device in row chunks, each block of QLD_OPT_BAND_ROWS rows is computed as
 * soon as the rows it needs have arrived, and its band rows are copied back
 * while the next block computes.  qLD has no band mode: its equivalent is a
 * split_region-style -inputList of window pairs (utilities/split_region),
 * one task each.
 */
int qld_cuda_ld_band(qld_ctx *ctx, const uint64_t *A, const uint32_t *bcA, int m, int K, int S,
                     int band, float *r2_band, uint32_t *counts_band);
/* Device-resident form: lda as in qld_ld_args, ldr/ldc >= band elements
 * between consecutive rows of the band arrays; asynchronous on `stream`. */
int qld_cuda_ld_band_device(qld_ctx *ctx, const uint64_t *A, const uint32_t *bcA, int m,
                            long long lda, int K, int S, int band, float *r2_band,
                            long long ldr, uint32_t *counts_band, long long ldc, void *stream);

/*
 * Many independent tasks (region pairs of any SNP and sample counts, single
 * or two-region) in ONE persistent launch: every output tile of every task is
 * a work item taken from a device work queue by the SMs as they free up.
 * Same per-task contract as qld_cuda_ld_device(); asynchronous on `stream`,
 * collect with qld_cuda_sync().  The tasks of one call must not overlap in
 * their outputs.  Each task gets the kernel qld_cuda_ld_device() would give
 * it (QLD_OPT_KERNEL, else the autotuner's entry for its shape class, else
 * the 4-bit kernel while K * 64 <= 2^24 and the popcount kernel past it):
 * the 4-bit tasks share the persistent launch, the others follow it on the
 * same stream as their own launches.  A forced kernel that is not exact for
 * a task returns QLD_ERR_UNSUPPORTED before anything runs.  qLD runs such task
 * lists one task at a time (-inputList: src/correlator/src/input_list.c:205-323,
 * correlate_function.c:59-83); this is their batched replacement.
 */
int qld_cuda_ld_batch(qld_ctx *ctx, const qld_ld_args *jobs, int njobs, void *stream);

/*
 * A batched call captured once as a CUDA graph and replayed.
 * qld_cuda_batch_plan checks and routes `jobs` exactly as qld_cuda_ld_batch()
 * does, builds their tensor maps and device job table once, and captures the
 * launch sequence (work-queue ticket reset, the persistent launch, the routed
 * tasks' own launches) into an executable graph; nothing runs.
 * qld_cuda_batch_run replays it on `stream` (NULL: the context's stream),
 * asynchronously: collect with qld_cuda_sync() as after qld_cuda_ld_batch().
 * The plan keeps the tasks' device pointers, so their tables, bit counts and
 * outputs must stay allocated while it lives; each replay reads the tables
 * as they are then (rewritten contents of the same shapes, e.g. resampled
 * haplotypes, need no new plan).  The context options in force when the plan
 * is made (r^2 mode, kernel choice, wait budget) hold for every replay.
 * Replays of one plan run one after another whatever their streams.
 * qld_cuda_batch_free waits for the plan's replays and frees it;
 * qld_cuda_release frees the plans still alive.  qLD has no equivalent: an
 * -inputList run re-reads and re-plans every task each time.
 */
typedef struct qld_batch_plan qld_batch_plan;
int qld_cuda_batch_plan(qld_ctx *ctx, const qld_ld_args *jobs, int njobs, qld_batch_plan **plan);
int qld_cuda_batch_run(qld_batch_plan *plan, void *stream);
int qld_cuda_batch_free(qld_batch_plan *plan);

/*
 * Serving: a request loop over chromosome tables resident in HBM.
 *
 * qld_srv_create starts a server on `device` with a device output pool of
 * `pool_bytes`; up to `max_inflight` batches run at once on their own
 * streams.  qld_srv_add_table copies a packed table (rows of K words, bit
 * counts, S samples) into HBM once.  qld_srv_submit enqueues a query -- SNP
 * rows [a0, a1) against rows [b0, b1) of one table (a single region when
 * the two ranges are equal, else all (a, b) pairs) -- and returns at once.
 * A worker thread admits pending queries in arrival order while their r^2
 * outputs ((b1-b0) x (a1-a0) floats) fit in the free pool, packs the
 * admitted ones into one persistent batched launch (qld_cuda_ld_batch's
 * kernel) and launches it while earlier batches still run: requests that
 * arrive while others are on the GPU join the next batch as slots and
 * memory free up (continuous batching).  Per query the server computes on
 * the device the pairs with threshold <= r^2 < 100 (the rows qLD's writer
 * would print at -r2limit threshold, correlate_IO.c:408), the sum of those
 * r^2 below 100 and their maximum.  If host_r2 is set the full r^2 block is
 * copied there and the device memory freed; otherwise it stays on the device
 * until qld_srv_release (qld_srv_fetch copies it).  qld_srv_poll returns
 * finished queries with their submit-to-ready latency.  No counterpart in
 * the reference (qLD-compute is a batch tool).
 */
typedef struct qld_server qld_server;

typedef struct qld_query {
    int table;
    int a0, a1;           /* side A: output columns (the reference's table A) */
    int b0, b1;           /* side B: output rows (table B) */
    float threshold;      /* summary threshold on r^2 */
    float *host_r2;       /* optional (b1-b0) x (a1-a0) host buffer */
} qld_query;

typedef struct qld_query_result {
    long long id;
    int status;           /* QLD_OK, or the error that ended the query */
    double latency_ms;    /* submit -> summary (and host_r2) ready */
    long long pairs;      /* r^2 values the query defines */
    long long n_above;    /* pairs with threshold <= r^2 < 100 */
    double sum_r2;        /* sum of r^2 < 100 (NaN excluded) */
    float max_r2;         /* largest r^2 < 100 (0 if none) */
} qld_query_result;

int qld_srv_create(int device, size_t pool_bytes, int max_inflight, qld_server **srv);
/* A and bc may be host or device pointers (K words per row, no padding).
 * The copy is synchronous but does not wait for work on other streams: a
 * device table written on a non-blocking stream must be complete first. */
int qld_srv_add_table(qld_server *srv, const uint64_t *A, const uint32_t *bc, int m, int K,
                      int S, int *table_id);
int qld_srv_submit(qld_server *srv, const qld_query *q, long long *id);
int qld_srv_poll(qld_server *srv, qld_query_result *out, int max, int *count, int wait_ms);
int qld_srv_fetch(qld_server *srv, long long id, float *host_r2);
int qld_srv_release(qld_server *srv, long long id);
int qld_srv_destroy(qld_server *srv);
const char *qld_srv_last_error(const qld_server *srv);

/* Pinned host memory for tables and results (the -cuda reader allocates its
 * tables here so the host<->device copies run asynchronously). */
int qld_cuda_host_alloc(qld_ctx *ctx, size_t bytes, void **ptr);
int qld_cuda_host_free(qld_ctx *ctx, void *ptr);

/* Counters since the last reset: counts-kernel launches, all launches of
 * this library's kernels, and (with QLD_OPT_PROFILE) the summed event time
 * of the counts-kernel launches in milliseconds. */
typedef struct qld_stats {
    long long counts_launches;
    long long kernel_launches;
    double counts_kernel_ms;
    int last_kernel;           /* QLD_KERNEL_* used by the last call */
    long long hits_rows;       /* qld_cuda_ld_hits: B rows delivered */
    long long hits_pairs;      /* qld_cuda_ld_hits: kept pairs delivered */
} qld_stats;

int qld_cuda_get_stats(qld_ctx *ctx, qld_stats *out, int reset);

/*
 * One LD task from host buffers that allocates nothing.  For callers that
 * cannot call cudaMalloc: a host program whose device memory is reserved
 * up front by another component (a pool or framework that owns the GPU's
 * memory), or a plug-in loaded into one.  Same arguments and result as
 * qld_cuda_ld() with r^2 in QLD_R2_EXACT mode and no counts output, on the
 * current device and the given stream (a cudaStream_t; NULL = the legacy
 * default stream); synchronous.  No context, stream, event or buffer is
 * created: all device memory it uses is one static scratch array of
 * QLD_NOALLOC_SCRATCH_BYTES that stays resident on every GPU where this code
 * is loaded until the process exits.  The first call on a device sets up the
 * array's device address; make that first call before any stream capture.
 * Limit: 256 + bit counts + the packed tables (rows x K rounded up to an
 * even word count x 8 bytes, A and, for two regions, B) plus at least one
 * r^2 band (min(n, 256) rows x m x 4 bytes) must fit in the scratch; larger
 * tasks return QLD_ERR_TOO_LARGE.  Calls share the scratch, so calls that
 * overlap on the GPU (two streams or two threads) race: serialize them.
 * On an error return nothing of the call is still running on the stream:
 * a failure after work was queued waits for that work first.
 * No counterpart in the reference.
 */
#define QLD_NOALLOC_SCRATCH_BYTES (16u << 20)
int qld_cuda_ld_noalloc(const uint64_t *A, const uint32_t *bcA, int m,
                        const uint64_t *B, const uint32_t *bcB, int n,
                        int K, int S, int symmetric, float *r2_out, void *stream);

/* Measured peak of the popcount pipe on this device, in bit-ops/s (one POPC
 * of an ANDed 32-bit word = 32 bit-ops): the compute roofline of the
 * QLD_KERNEL_POPC variant.  Runs a register-only kernel for ~0.1 s.
 * No counterpart in the reference (its roofline is not measured). */
int qld_cuda_measure_popc_peak(qld_ctx *ctx, double *bitops_per_s);
/* The tensor pipe's dense rate for kernel QLD_KERNEL_MMA (kind::i8) or
 * QLD_KERNEL_FP4 (kind::mxf4) in operations (2 per multiply-accumulate) per
 * second: back-to-back 128 x 256 MMAs on a fixed tile, one CTA per SM.  The
 * denominator of those kernels' roofline.  Runs ~10 ms. */
int qld_cuda_measure_mma_peak(qld_ctx *ctx, int kernel, double *ops_per_s);

/*
 * Autotuner: measures every counts kernel that is exact for the shape
 * (popcount; int8 MMA with 128- and 256-row tiles while K * 64 <= 131,071;
 * 4-bit MMA on single SMs and on SM pairs while K * 64 <= 2^24) on a
 * synthetic task of m x n SNPs (n = m when `symmetric`) and K words, and
 * records the fastest for the task's shape class: floor(log2) of m, n and K,
 * single versus two regions, and the context's r^2 mode (tune once per mode
 * used).  From then on QLD_KERNEL_AUTO uses the
 * recorded kernel and tile option for tasks of that class (explicit
 * QLD_OPT_MMA_TILE / QLD_OPT_SM_PAIR values still win; band tasks and
 * untuned classes keep the built-in rule: the 4-bit kernel on SM pairs
 * while exact, else popcount).  Sides above 16,384 are measured at 16,384.
 * Outputs (each may be NULL): the kernel (QLD_KERNEL_*), its tile option
 * (MMA tile rows, SMs per 4-bit tile, 0 for popcount) and the time of one
 * launch in ms.  Uses the context's device buffers; synchronous.  No
 * counterpart in the reference, which fixes its BLIS micro-kernel and
 * blocking at build time (src/correlator/include/header.h:80-87).
 */
int qld_cuda_autotune(qld_ctx *ctx, int m, int n, int K, int symmetric, int *kernel,
                      int *option, float *ms);
/* The tuning table as text ("qld-tune 1", then one line per shape class:
 * log2 m, log2 n, log2 K, kind (0 two regions, 1 single region, +4 in
 * QLD_R2_REFERENCE mode), kernel, option, ms).  Loading
 * adds to (and overrides entries of) the context's table; a malformed file
 * changes nothing and returns QLD_ERR_INVALID. */
int qld_cuda_tune_save(qld_ctx *ctx, const char *path);
int qld_cuda_tune_load(qld_ctx *ctx, const char *path);

#ifdef __cplusplus
}
#endif

#endif /* QLD_CUDA_H */
