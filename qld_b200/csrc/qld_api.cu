// qld_api.cu -- the C ABI of libqld_cuda (declared in include/qld_cuda.h).
//
// Host-buffer calls (qld_cuda_ld) stage the packed tables into device memory
// with one pitched copy each (the device pitch is K rounded up to an even
// word count so every row starts 16-byte aligned for TMA), then walk the B
// rows in bands: band t's kernel writes its r^2 rows into one of two device
// band buffers while the copy stream moves band t-1's rows to the caller's
// buffer, so the device->host stream overlaps the counts kernels.
#include <cudaTypedefs.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

#include "qld_cuda.h"
#include "qld_kernels.h"
#include "tcgen05.cuh"

using namespace qld;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct HostBuf {   // pinned
    void *p = nullptr;
    size_t bytes = 0;
};

// One autotuned choice of counts kernel: the variant, its tile option
// (QLD_OPT_MMA_TILE rows for the int8 kernels, QLD_OPT_SM_PAIR SMs per tile
// for the 4-bit kernel, 0 for popc) and the measured time per launch.
struct TuneChoice {
    int kernel, option;
    float ms;
};

}  // namespace

struct qld_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;   // kernels and host->device copies
    cudaStream_t copy = nullptr;     // device->host result copies
    cudaStream_t h2d = nullptr;      // chunked host->device table copies (band calls)
    std::vector<cudaEvent_t> h2d_ev;
    unsigned *d_status = nullptr;
    unsigned *h_status = nullptr;    // pinned mirror of d_status
    char err[512] = {0};
    int kernel = QLD_KERNEL_AUTO;
    int r2_mode = QLD_R2_EXACT;
    int profile = 0;
    int band_rows = 4096;
    int mma_tile = 0;                 // 0: per shape, else 128 or 256
    int sm_pair = 0;                  // 4-bit kernel: 0 per shape, 1 or 2 SMs per tile
    std::map<long long, TuneChoice> tune;   // qld_cuda_autotune results by shape class
    long long timeout_cycles = 4000000000LL;  // ~2 s at boost clock
    size_t mem_cap = 0;               // QLD_OPT_MEM_CAP: 0 = no cap
    size_t mem_held = 0;              // bytes of the buffers ensure() holds
    DevBuf dA, dB, dbcA, dbcB, dOut[2], dCnt[2];
    DevBuf dStage;                    // host rows of odd K before padding (upload_rows)
    DevBuf dJobs, dQueue;             // batched launches: job table, ticket counter
    std::vector<BatchJob> hJobs;
    cudaEvent_t ev_band[2] = {nullptr, nullptr};
    cudaEvent_t ev_copy[2] = {nullptr, nullptr};
    // qld_cuda_ld_hits: per slot the device mask / counts / offsets / values
    // and their pinned host mirrors
    DevBuf dMask[2], dHcnt[2], dHoff[2], dHval[2];
    HostBuf hMask[2], hOff[2], hVal[2], hStat;
    // qld_cuda_vcf_pack
    DevBuf vText, vSites, vValid, vSlash, vRoff, vRnd, vScratch, vWords, vBc, vLen, vKeep, vErr;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof;
    size_t prof_used = 0;
    bool capturing = false;           // a batch plan is being captured: no profiling events
    std::vector<qld_batch_plan *> plans;   // live plans, freed by qld_cuda_release
    qld_stats stats{};
    PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
};

// A batched call captured once: its device job table and ticket counter, and
// the executable graph of its launch sequence.
struct qld_batch_plan {
    qld_ctx *ctx = nullptr;
    BatchJob *d_jobs = nullptr;
    unsigned long long *d_queue = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;   // null: the plan has no work
    cudaEvent_t done = nullptr;       // recorded after every replay
    long long counts_launches = 0, kernel_launches = 0;   // per replay
    int last_kernel = 0;
};

namespace {

int set_err(qld_ctx *c, int code, const char *fmt, ...) {
    if (c) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(c->err, sizeof c->err, fmt, ap);
        va_end(ap);
    }
    return code;
}

#define CUDA_TRY(ctx, expr)                                                              \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return set_err((ctx), QLD_ERR_CUDA, "%s failed: %s", #expr,                  \
                           cudaGetErrorString(e_));                                      \
    } while (0)

int ensure(qld_ctx *c, DevBuf &b, size_t bytes) {
    if (bytes <= b.bytes) return QLD_OK;
    const size_t others = c->mem_held - b.bytes;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    c->mem_held = others;
    if (c->mem_cap && others + bytes > c->mem_cap)
        return set_err(c, QLD_ERR_NOMEM,
                       "device memory cap: %zu bytes held + %zu needed > cap of %zu", others,
                       bytes, c->mem_cap);
    size_t want = bytes + bytes / 8;  // headroom so nearby sizes reuse the buffer
    if (c->mem_cap && others + want > c->mem_cap) want = bytes;
    if (cudaMalloc(&b.p, want) != cudaSuccess) {
        cudaGetLastError();
        if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            return set_err(c, QLD_ERR_NOMEM, "cudaMalloc(%zu) failed", bytes);
        }
        want = bytes;
    }
    b.bytes = want;
    c->mem_held = others + want;
    return QLD_OK;
}

int ensure_host(qld_ctx *c, HostBuf &b, size_t bytes) {
    if (bytes <= b.bytes) return QLD_OK;
    if (b.p) cudaFreeHost(b.p);
    b.p = nullptr;
    b.bytes = 0;
    const size_t want = bytes + bytes / 4;
    if (cudaMallocHost(&b.p, want) != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return set_err(c, QLD_ERR_NOMEM, "cudaMallocHost(%zu) failed", want);
    }
    b.bytes = want;
    return QLD_OK;
}

// Tensor map over a row-major table of `rows` rows, K uint64 words used per
// row, `ld` words between rows; box = box_words x box_rows, 128-byte swizzle.
int make_tmap(qld_ctx *c, CUtensorMap *tm, const void *base, int rows, int K, long long ld,
              int box_words, int box_rows, int swizzle) {
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
    cuuint32_t box[2] = {(cuuint32_t)box_words, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    const CUtensorMapSwizzle sw =
        swizzle == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
    CUresult r = c->encode(tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void *>(base), dims,
                           strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return set_err(c, QLD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d): rows=%d K=%d ld=%lld",
                       (int)r, rows, K, ld);
    return QLD_OK;
}

struct Task {
    const uint64_t *A; const uint32_t *bcA; int m; long long lda;
    const uint64_t *B; const uint32_t *bcB; int n; long long ldb;
    int K, S, symmetric;
    int band;   // > 0: single region, entries 1 <= a - b <= band only
};

bool mma_exact_for(const Task &t) { return (long long)t.K * 64 <= kMmaMaxSamples; }
bool fp4_exact_for(const Task &t) { return (long long)t.K * 64 <= kMxf4MaxSamples; }

// Shape class of a task for the autotuner's table: floor(log2) of m, n and
// K, and the kind (0 two regions, 1 single region, 2 band; +4 in
// R2_REFERENCE mode, whose epilogue changes which kernel is fastest).  Tasks
// in one class differ in size by less than 2x on every side.
int ilog2(long long x) {
    int r = 0;
    while (x > 1) { x >>= 1; ++r; }
    return r;
}
long long tune_key(int m, int n, int K, int kind) {
    return ((long long)ilog2(m) << 24) | ((long long)ilog2(n) << 16) |
           ((long long)ilog2(K) << 8) | (long long)kind;
}
int task_kind(const Task &t, int r2_mode) {
    return (t.band > 0 ? 2 : (t.symmetric ? 1 : 0)) + (r2_mode == QLD_R2_REFERENCE ? 4 : 0);
}

bool exact_for(int kernel, const Task &t);

// The autotuned choice for the task's shape class, when the kernel option is
// automatic, the class was tuned, and the tuned kernel is exact for the task.
const TuneChoice *tuned_for(qld_ctx *c, const Task &t) {
    if (c->kernel != QLD_KERNEL_AUTO || c->tune.empty()) return nullptr;
    auto it = c->tune.find(tune_key(t.m, t.n, t.K, task_kind(t, c->r2_mode)));
    if (it == c->tune.end() || !exact_for(it->second.kernel, t)) return nullptr;
    return &it->second;
}

// Per-shape variant: the 4-bit tensor-core kernel wherever its F32
// accumulators stay exact (K * 64 <= 2^24 samples: measured faster than the
// i8 kernels on large and small tasks alike), the popcount kernel otherwise.
int choose_kernel(qld_ctx *c, const Task &t) {
    if (const TuneChoice *tc = tuned_for(c, t)) return tc->kernel;
    return fp4_exact_for(t) ? QLD_KERNEL_FP4 : QLD_KERNEL_POPC;
}

bool exact_for(int kernel, const Task &t) {
    if (kernel == QLD_KERNEL_MMA) return mma_exact_for(t);
    if (kernel == QLD_KERNEL_FP4) return fp4_exact_for(t);
    return kernel == QLD_KERNEL_POPC;
}

long long tile_count(const Task &t, int bm, int bn, int b0, int b1) {
    const int tb0 = b0 / bn, tiles_b = (b1 - b0 + bn - 1) / bn;
    if (bm == 256 && bn == 240)
        return tc::TileList<256, 240>{(t.m + 255) / 256, tb0, tiles_b, t.symmetric, t.band}.count();
    if (bm == 128 && bn == 240)
        return tc::TileList<128, 240>{(t.m + 127) / 128, tb0, tiles_b, t.symmetric, t.band}.count();
    if (bm == 256 && bn == 256)
        return tc::TileList<256, 256>{(t.m + 255) / 256, tb0, tiles_b, t.symmetric, t.band}.count();
    if (bm == 128 && bn == 256)
        return tc::TileList<128, 256>{(t.m + 127) / 128, tb0, tiles_b, t.symmetric, t.band}.count();
    return tc::TileList<128, 128>{(t.m + 127) / 128, tb0, tiles_b, t.symmetric, t.band}.count();
}

// The 256 x 256 tile unpacks 2/3 of the bytes per multiply-accumulate but
// cannot overlap its epilogue; it pays off once there are enough tiles to
// keep every SM busy for several rounds.
const KernelShape &mma_shape(qld_ctx *c, const Task &t, int b0, int b1) {
    if (c->mma_tile == 128) return kMmaShape;
    if (c->mma_tile == 256) return kMmaWideShape;
    if (const TuneChoice *tc = tuned_for(c, t))
        if (tc->kernel == QLD_KERNEL_MMA) return tc->option == 256 ? kMmaWideShape : kMmaShape;
    return tile_count(t, 256, 256, b0, b1) >= 4LL * c->sm_count ? kMmaWideShape : kMmaShape;
}

// The 4-bit kernel on SM pairs or single SMs (same 256 x 240 tiles).  The
// pair kernel overlaps each tile's epilogue with the next tile's MMAs and
// finishes a tile on two SMs in half the time: the faster one in both r^2
// modes (a single region of 29,817 SNPs x 16,622 samples: 2.40 against
// 3.16 ms exact, 2.63 against 4.14 ms reference).
const KernelShape &fp4_shape(qld_ctx *c, const Task &t, int b0, int b1) {
    (void)b0; (void)b1;
    if (c->sm_pair == 0)
        if (const TuneChoice *tc = tuned_for(c, t))
            if (tc->kernel == QLD_KERNEL_FP4) return tc->option == 1 ? kMxf4Shape : kMxf4PairShape;
    return c->sm_pair == 1 ? kMxf4Shape : kMxf4PairShape;
}

const KernelShape &shape_of(qld_ctx *c, int variant, const Task &t, int b0, int b1) {
    if (variant == QLD_KERNEL_FP4) return fp4_shape(c, t, b0, b1);
    return variant == QLD_KERNEL_MMA ? mma_shape(c, t, b0, b1) : kPopcShape;
}

int variant_of(qld_ctx *c, const Task &t) {
    return c->kernel == QLD_KERNEL_AUTO ? choose_kernel(c, t) : c->kernel;
}

// B rows per streamed band: the context's band size rounded down to whole
// tile rows of the task's kernel (240 for the 4-bit kernel, else 256).
int band_rows_for(qld_ctx *c, const Task &t) {
    const int unit = variant_of(c, t) == QLD_KERNEL_FP4 ? kMxf4Shape.bn : 256;
    const int b = c->band_rows / unit * unit;
    return b > unit ? b : unit;
}

// With QLD_OPT_PROFILE: an event pair around the next launch on `st`
// (*end receives the closing event, recorded by the caller after the launch).
int prof_begin(qld_ctx *c, cudaStream_t st, cudaEvent_t *end) {
    *end = nullptr;
    if (!c->profile || c->capturing) return QLD_OK;
    if (c->prof_used == c->prof.size()) {
        cudaEvent_t a, b;
        CUDA_TRY(c, cudaEventCreate(&a));
        CUDA_TRY(c, cudaEventCreate(&b));
        c->prof.emplace_back(a, b);
    }
    *end = c->prof[c->prof_used].second;
    CUDA_TRY(c, cudaEventRecord(c->prof[c->prof_used].first, st));
    ++c->prof_used;
    return QLD_OK;
}

// Launch the counts kernel over B rows [b0, b1) (b0 a multiple of the
// kernel's tile rows: band_rows_for), writing r2/counts rows relative to
// out_row0.
int launch_counts(qld_ctx *c, const Task &t, int b0, int b1, float *r2, long long ldr,
                  uint32_t *cnt, long long ldc, int out_row0, cudaStream_t st) {
    const int variant = variant_of(c, t);
    if (variant == QLD_KERNEL_MMA && !mma_exact_for(t))
        return set_err(c, QLD_ERR_UNSUPPORTED,
                       "tensor-core kernel needs K*64 <= %d samples (K=%d)", kMmaMaxSamples, t.K);
    if (variant == QLD_KERNEL_FP4 && !fp4_exact_for(t))
        return set_err(c, QLD_ERR_UNSUPPORTED,
                       "4-bit tensor-core kernel needs K*64 <= %d samples (K=%d)",
                       kMxf4MaxSamples, t.K);
    const KernelShape &ks = shape_of(c, variant, t, b0, b1);
    CUtensorMap tmA, tmB;
    int rc;
    if ((rc = make_tmap(c, &tmA, t.A, t.m, t.K, t.lda, ks.box_words, ks.box_rows_a, ks.swizzle)) ||
        (rc = make_tmap(c, &tmB, t.B, t.n, t.K, t.ldb, ks.box_words, ks.box_rows_b, ks.swizzle)))
        return rc;
    const int tb0 = b0 / ks.bn;
    const int tiles_b = (b1 - b0 + ks.bn - 1) / ks.bn;
    LdParams p{};
    p.m = t.m; p.n = t.n; p.K = t.K; p.S = t.S;
    p.symmetric = t.symmetric;
    p.band = t.band;
    p.nk = (t.K + ks.box_words - 1) / ks.box_words;
    p.bcA = t.bcA; p.bcB = t.bcB;
    p.r2 = r2; p.ldr = ldr; p.counts = cnt; p.ldc = ldc; p.out_row0 = out_row0;
    if (t.band > 0) {
        // Band array: entry (b, a) at r2[(b - out_row0) * ldr + (a - b - 1)], i.e. the
        // kernels' (b - out_row0) * ldr' + a with ldr' = ldr - 1 and a shifted base.
        p.r2 = r2 - out_row0 - 1;
        p.ldr = ldr - 1;
        if (cnt) { p.counts = cnt - out_row0 - 1; p.ldc = ldc - 1; }
    }
    p.status = c->d_status;
    p.timeout_cycles = c->timeout_cycles;
    for (int done = 0; done < tiles_b; done += 65535) {
        const int nb = tiles_b - done < 65535 ? tiles_b - done : 65535;
        p.tb0 = tb0 + done;
        cudaEvent_t e1 = nullptr;
        if (int rc = prof_begin(c, st, &e1)) return rc;
        cudaError_t e =
            &ks == &kMxf4PairShape    ? launch_mxf4_pair(tmA, tmB, p, nb, c->r2_mode, st)
            : variant == QLD_KERNEL_FP4 ? launch_mxf4(tmA, tmB, p, nb, c->r2_mode, st)
            : variant != QLD_KERNEL_MMA ? launch_popc(tmA, tmB, p, nb, c->r2_mode, st)
            : &ks == &kMmaWideShape     ? launch_mma_wide(tmA, tmB, p, nb, c->r2_mode, st)
                                        : launch_mma(tmA, tmB, p, nb, c->r2_mode, st);
        if (e != cudaSuccess)
            return set_err(c, QLD_ERR_CUDA, "counts kernel launch failed: %s", cudaGetErrorString(e));
        if (e1) CUDA_TRY(c, cudaEventRecord(e1, st));
        c->stats.counts_launches++;
        c->stats.kernel_launches++;
    }
    c->stats.last_kernel = variant;
    return QLD_OK;
}

// Wait for `st`, fold the profiled kernel times in, and read/clear the status.
int finish(qld_ctx *c, cudaStream_t st) {
    CUDA_TRY(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(unsigned),
                                cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    for (size_t i = 0; i < c->prof_used; ++i) {
        float ms = 0.f;
        CUDA_TRY(c, cudaEventElapsedTime(&ms, c->prof[i].first, c->prof[i].second));
        c->stats.counts_kernel_ms += ms;
    }
    c->prof_used = 0;
    const unsigned st_bits = *c->h_status;
    if (st_bits) {
        CUDA_TRY(c, cudaMemsetAsync(c->d_status, 0, sizeof(unsigned), st));
        CUDA_TRY(c, cudaStreamSynchronize(st));
        return set_err(c, QLD_ERR_TIMEOUT, "a counts kernel gave up a bounded wait (status 0x%x)",
                       st_bits);
    }
    return QLD_OK;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// COUNTSTATES over B rows [b0, b1) (b0 a multiple of 128), one byte per pair
// at out[(b - out_row0) * lds + a].
int launch_states_range(qld_ctx *c, const Task &t, int b0, int b1, uint8_t *out, long long lds,
                        int out_row0, cudaStream_t st) {
    const KernelShape &ks = kStatesShape;
    CUtensorMap tmA, tmB;
    int rc;
    if ((rc = make_tmap(c, &tmA, t.A, t.m, t.K, t.lda, ks.box_words, ks.box_rows_a, ks.swizzle)) ||
        (rc = make_tmap(c, &tmB, t.B, t.n, t.K, t.ldb, ks.box_words, ks.box_rows_b, ks.swizzle)))
        return rc;
    const int tb0 = b0 / ks.bn;
    const int tiles_b = (b1 - b0 + ks.bn - 1) / ks.bn;
    StatesParams p{};
    p.m = t.m; p.n = t.n; p.K = t.K; p.symmetric = t.symmetric;
    p.out = out; p.lds = lds; p.out_row0 = out_row0;
    p.status = c->d_status;
    p.timeout_cycles = c->timeout_cycles;
    for (int done = 0; done < tiles_b; done += 65535) {
        const int nb = tiles_b - done < 65535 ? tiles_b - done : 65535;
        p.tb0 = tb0 + done;
        cudaEvent_t e1 = nullptr;
        if ((rc = prof_begin(c, st, &e1))) return rc;
        cudaError_t e = launch_states(tmA, tmB, p, nb, st);
        if (e != cudaSuccess)
            return set_err(c, QLD_ERR_CUDA, "states kernel launch failed: %s",
                           cudaGetErrorString(e));
        if (e1) CUDA_TRY(c, cudaEventRecord(e1, st));
        c->stats.kernel_launches++;
    }
    return QLD_OK;
}

// Rows of odd K go through the staging buffer this many at a time, so it
// stays small next to the tables themselves.
constexpr long long kStageRows = 8192;

// Host rows of K words -> device rows of ldd words (ldd = K, or K + 1 to
// keep rows 16-byte aligned).  A row-pitched 2-D copy moves rows of a few KB
// at about a third of the link rate (19 vs 55 GB/s for 2,080-byte rows on a
// B200) and slows device->host copies running beside it to a crawl, so the
// rows go up as 1-D copies: in place when ldd == K, else kStageRows at a
// time into `stage` (reused in stream order) and a kernel spreads them to
// the padded pitch.
int upload_rows(qld_ctx *c, uint64_t *dst, long long ldd, const uint64_t *src, int K,
                long long rows, uint64_t *stage, cudaStream_t st) {
    if (rows <= 0) return QLD_OK;
    if (ldd == K) {
        CUDA_TRY(c, cudaMemcpyAsync(dst, src, (size_t)rows * K * 8, cudaMemcpyHostToDevice, st));
        return QLD_OK;
    }
    for (long long r0 = 0; r0 < rows; r0 += kStageRows) {
        const long long nr = rows - r0 < kStageRows ? rows - r0 : kStageRows;
        CUDA_TRY(c, cudaMemcpyAsync(stage, src + r0 * K, (size_t)nr * K * 8,
                                    cudaMemcpyHostToDevice, st));
        const cudaError_t e = launch_pad_rows(dst + r0 * ldd, ldd, stage, K, nr, st);
        if (e != cudaSuccess)
            return set_err(c, QLD_ERR_CUDA, "row padding launch failed: %s",
                           cudaGetErrorString(e));
        c->stats.kernel_launches++;
    }
    return QLD_OK;
}

// The staging buffer upload_rows needs for tables of up to `rows` rows
// (none for even K).
int ensure_stage(qld_ctx *c, int K, long long rows, uint64_t **stage) {
    *stage = nullptr;
    if (!(K & 1)) return QLD_OK;
    const long long r = rows < kStageRows ? rows : kStageRows;
    if (int rc = ensure(c, c->dStage, (size_t)r * K * 8)) return rc;
    *stage = static_cast<uint64_t *>(c->dStage.p);
    return QLD_OK;
}

// Copy host tables into the context's device buffers (rows padded to an even
// word count, 16-byte aligned for TMA) on c->stream; *t describes them.
// NULL bit counts are not copied (COUNTSTATES does not use them).
int stage_tables(qld_ctx *c, const uint64_t *A, const uint32_t *bcA, int m, const uint64_t *B,
                 const uint32_t *bcB, int n, int K, int S, int symmetric, Task *t) {
    const long long Kp = K + (K & 1);
    int rc;
    if ((rc = ensure(c, c->dA, (size_t)m * Kp * 8)) || (rc = ensure(c, c->dbcA, (size_t)m * 4)))
        return rc;
    uint64_t *stage;
    if ((rc = ensure_stage(c, K, symmetric || n < m ? m : n, &stage))) return rc;
    if ((rc = upload_rows(c, static_cast<uint64_t *>(c->dA.p), Kp, A, K, m, stage, c->stream)))
        return rc;
    if (bcA)
        CUDA_TRY(c, cudaMemcpyAsync(c->dbcA.p, bcA, (size_t)m * 4, cudaMemcpyHostToDevice,
                                    c->stream));
    const uint64_t *dB = static_cast<const uint64_t *>(c->dA.p);
    const uint32_t *dbcB = static_cast<const uint32_t *>(c->dbcA.p);
    if (!symmetric) {
        if ((rc = ensure(c, c->dB, (size_t)n * Kp * 8)) || (rc = ensure(c, c->dbcB, (size_t)n * 4)))
            return rc;
        if ((rc = upload_rows(c, static_cast<uint64_t *>(c->dB.p), Kp, B, K, n, stage,
                              c->stream)))
            return rc;
        if (bcB)
            CUDA_TRY(c, cudaMemcpyAsync(c->dbcB.p, bcB, (size_t)n * 4, cudaMemcpyHostToDevice,
                                        c->stream));
        dB = static_cast<const uint64_t *>(c->dB.p);
        dbcB = static_cast<const uint32_t *>(c->dbcB.p);
    }
    *t = Task{static_cast<const uint64_t *>(c->dA.p), static_cast<const uint32_t *>(c->dbcA.p), m,
              Kp, dB, dbcB, n, Kp, K, S, symmetric, 0};
    return QLD_OK;
}

}  // namespace

// ================================================================== C ABI ==

namespace {

// Autotuner inputs: pseudo-random packed rows (splitmix64 of the word index,
// zero past word K) and their bit counts, so the tuned kernels run on
// consistent data.
__global__ void k_tune_fill(uint64_t *T, long long rows, int K, long long ld, uint64_t seed) {
    const long long n = rows * ld;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        uint64_t z = seed + (uint64_t)i * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        T[i] = (i % ld) < K ? (z ^ (z >> 31)) : 0ull;
    }
}

__global__ void k_tune_bc(const uint64_t *T, long long rows, int K, long long ld, uint32_t *bc) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows;
         r += (long long)gridDim.x * blockDim.x) {
        uint32_t c = 0;
        for (int w = 0; w < K; ++w) c += (uint32_t)__popcll(T[r * ld + w]);
        bc[r] = c;
    }
}

// Puts the context's kernel options and statistics back when the tuner
// returns, on every path.
struct OptionGuard {
    qld_ctx *c;
    int kernel, mma_tile, sm_pair;
    qld_stats stats;
    explicit OptionGuard(qld_ctx *ctx)
        : c(ctx), kernel(ctx->kernel), mma_tile(ctx->mma_tile), sm_pair(ctx->sm_pair),
          stats(ctx->stats) {}
    ~OptionGuard() {
        c->kernel = kernel;
        c->mma_tile = mma_tile;
        c->sm_pair = sm_pair;
        c->stats = stats;
    }
};

constexpr int kTuneMaxSide = 16384;   // the tuner measures at most 16,384 x 16,384

// Part `part` of `nparts` of a task's B rows for a split over GPUs:
// consecutive whole B tile rows of the kernel's tiles, with (nearly) equal
// numbers of output tiles -- equal bit-ops, since every tile of a task costs
// K words.  Part k starts at the first tile row before which k/nparts of the
// task's tiles lie; trailing parts of a task with fewer tile rows than parts
// are empty (row0 == row1).
void split_rows(const Task &t, int bm, int bn, int part, int nparts, int *r0, int *r1) {
    const int nb = (t.n + bn - 1) / bn;
    const long long total = tile_count(t, bm, bn, 0, t.n);
    auto boundary = [&](int k) -> int {
        if (k <= 0) return 0;
        if (k >= nparts) return t.n;
        const long long target = total * k / nparts;
        long long cum = 0;
        for (int tb = 0; tb < nb; ++tb) {
            if (cum >= target) return tb * bn;
            const int e = (tb + 1) * bn < t.n ? (tb + 1) * bn : t.n;
            cum += tile_count(t, bm, bn, tb * bn, e);
        }
        return t.n;
    };
    *r0 = boundary(part);
    *r1 = boundary(part + 1);
}

const KernelShape &split_shape(int variant) {
    return variant == QLD_KERNEL_FP4 ? kMxf4PairShape
           : variant == QLD_KERNEL_MMA ? kMmaShape : kPopcShape;
}

// A batched task that runs as its own launch (not the 4-bit kernel, or past
// 2^24 samples), with its outputs.
struct RoutedTask {
    Task t;
    float *r2;
    long long ldr;
    uint32_t *counts;
    long long ldc;
};

// The host half of a batched call: checks every task, routes it (the kernel
// qld_cuda_ld_device would give it), and fills `hj` with the job table of the
// 4-bit tasks -- tensor maps built, most expensive first so the queue ends on
// small items -- and `routed` with the others.  `items` = output tiles of hj.
int prepare_batch(qld_ctx *c, const qld_ld_args *jobs, int njobs, std::vector<BatchJob> &hj,
                  std::vector<RoutedTask> &routed, long long &items) {
    const KernelShape &ks = kBatchShape;
    std::vector<long long> tiles(njobs), cost(njobs);
    std::vector<int> order;
    order.reserve(njobs);
    routed.clear();
    for (int j = 0; j < njobs; ++j) {
        qld_ld_args a = jobs[j];
        if (a.symmetric) { a.B = a.A; a.bcB = a.bcA; a.n = a.m; a.ldb = a.lda; }
        if (a.m < 0 || a.n < 0 || a.K < 1 || a.S < 1 || a.lda < a.K || a.ldb < a.K ||
            (a.lda & 1) || (a.ldb & 1) || a.ldr < a.m || (a.counts && a.ldc < a.m) || !a.A ||
            !a.B || !a.bcA || !a.bcB || !a.r2 || !aligned16(a.A) || !aligned16(a.B))
            return set_err(c, QLD_ERR_INVALID, "batch job %d: bad sizes, strides or pointers", j);
        Task t{a.A, a.bcA, a.m, a.lda, a.B, a.bcB, a.n, a.ldb, a.K, a.S, a.symmetric, 0};
        const int variant = variant_of(c, t);
        if (!exact_for(variant, t))
            return set_err(c, QLD_ERR_UNSUPPORTED,
                           "batch job %d: the forced kernel is not exact for K*64 = %lld samples",
                           j, (long long)a.K * 64);
        tiles[j] = (a.m == 0 || a.n == 0) ? 0 : tile_count(t, ks.bm, ks.bn, 0, a.n);
        if (variant != QLD_KERNEL_FP4 || (long long)a.K * 64 > kBatchMaxSamples) {
            if (tiles[j] > 0) routed.push_back({t, a.r2, a.ldr, a.counts, a.ldc});
            continue;
        }
        cost[j] = tiles[j] * (long long)a.K;
        order.push_back(j);
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return cost[x] > cost[y]; });
    const int nb = (int)order.size();
    hj.resize(nb);
    items = 0;
    for (int i = 0; i < nb; ++i) {
        const int j = order[i];
        qld_ld_args a = jobs[j];
        if (a.symmetric) { a.B = a.A; a.bcB = a.bcA; a.n = a.m; a.ldb = a.lda; }
        BatchJob &J = hj[i];
        memset(&J, 0, sizeof J);
        J.bcA = a.bcA; J.bcB = a.bcB; J.r2 = a.r2; J.counts = a.counts;
        J.ldr = a.ldr; J.ldc = a.ldc; J.item0 = items;
        J.m = a.m; J.n = a.n; J.K = a.K; J.S = a.S; J.symmetric = a.symmetric;
        if (tiles[j] > 0) {
            int rc;
            if ((rc = make_tmap(c, &J.tmA, a.A, a.m, a.K, a.lda, ks.box_words, ks.box_rows_a,
                                ks.swizzle)) ||
                (rc = make_tmap(c, &J.tmB, a.B, a.n, a.K, a.ldb, ks.box_words, ks.box_rows_b,
                                ks.swizzle)))
                return rc;
        }
        items += tiles[j];
    }
    return QLD_OK;
}

// The launch sequence of a batched call on `st`: ticket reset and the
// persistent launch over the nb jobs at d_jobs (when they have items), then
// the routed tasks' own launches.
int enqueue_batch(qld_ctx *c, const BatchJob *d_jobs, int nb, long long items,
                  unsigned long long *d_queue, const std::vector<RoutedTask> &routed,
                  cudaStream_t st) {
    int rc;
    if (items > 0) {
        CUDA_TRY(c, cudaMemsetAsync(d_queue, 0, sizeof(unsigned long long), st));
        BatchParams bp{};
        bp.jobs = d_jobs;
        bp.njobs = nb;
        bp.nitems = items;
        bp.queue = d_queue;
        bp.status = c->d_status;
        bp.timeout_cycles = c->timeout_cycles;
        cudaEvent_t e1 = nullptr;
        if ((rc = prof_begin(c, st, &e1))) return rc;
        cudaError_t e = launch_batch(bp, c->r2_mode, 0, st);
        if (e != cudaSuccess)
            return set_err(c, QLD_ERR_CUDA, "batched launch failed: %s", cudaGetErrorString(e));
        if (e1) CUDA_TRY(c, cudaEventRecord(e1, st));
        c->stats.counts_launches++;
        c->stats.kernel_launches++;
        c->stats.last_kernel = QLD_KERNEL_FP4;
    }
    for (const RoutedTask &r : routed)
        if ((rc = launch_counts(c, r.t, 0, r.t.n, r.r2, r.ldr, r.counts, r.ldc, 0, st)))
            return rc;
    return QLD_OK;
}

void destroy_plan(qld_batch_plan *p) {
    if (p->done) cudaEventSynchronize(p->done);   // replays still in flight
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->done) cudaEventDestroy(p->done);
    if (p->d_jobs) cudaFree(p->d_jobs);
    if (p->d_queue) cudaFree(p->d_queue);
    delete p;
}

// Upload the plan's job table and capture its launch sequence (relaxed
// capture mode: the launchers' attribute and occupancy queries are not
// stream work) into an executable graph.  The capture's launches are not
// counted in the statistics; every replay adds them.
int build_plan(qld_ctx *c, qld_batch_plan *p, const std::vector<BatchJob> &hj, long long items,
               const std::vector<RoutedTask> &routed) {
    if (items == 0 && routed.empty()) return QLD_OK;
    const size_t jb = sizeof(BatchJob) * (hj.empty() ? 1 : hj.size());
    if (cudaMalloc(&p->d_jobs, jb) != cudaSuccess ||
        cudaMalloc(&p->d_queue, sizeof(unsigned long long)) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, QLD_ERR_NOMEM, "batch plan: cudaMalloc of the job table failed");
    }
    if (!hj.empty())
        CUDA_TRY(c, cudaMemcpy(p->d_jobs, hj.data(), sizeof(BatchJob) * hj.size(),
                               cudaMemcpyHostToDevice));
    CUDA_TRY(c, cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming));
    cudaStream_t cs = nullptr;
    CUDA_TRY(c, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    const qld_stats saved = c->stats;
    int rc = QLD_OK;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        c->capturing = true;
        rc = enqueue_batch(c, p->d_jobs, (int)hj.size(), items, p->d_queue, routed, cs);
        c->capturing = false;
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(cs, &g);   // ends the capture on every path
        p->graph = g;
    }
    p->counts_launches = c->stats.counts_launches - saved.counts_launches;
    p->kernel_launches = c->stats.kernel_launches - saved.kernel_launches;
    p->last_kernel = c->stats.last_kernel;
    c->stats = saved;
    cudaStreamDestroy(cs);
    if (rc) return rc;
    if (e != cudaSuccess || !p->graph)
        return set_err(c, QLD_ERR_CUDA, "batch plan: stream capture failed: %s",
                       cudaGetErrorString(e));
    CUDA_TRY(c, cudaGraphInstantiate(&p->exec, p->graph, 0));
    return QLD_OK;
}

}  // namespace

extern "C" {

int qld_cuda_init(int device, qld_ctx **ctx_out) {
    if (!ctx_out) return QLD_ERR_INVALID;
    *ctx_out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return QLD_ERR_NODEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10)
        return QLD_ERR_NODEVICE;
    qld_ctx *c = new (std::nothrow) qld_ctx();
    if (!c) return QLD_ERR_NOMEM;
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    if (const char *s = getenv("QLD_TIMEOUT_CYCLES")) c->timeout_cycles = atoll(s);
    int rc = QLD_OK;
    do {
        if (cudaSetDevice(device) != cudaSuccess) { rc = QLD_ERR_CUDA; break; }
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking) != cudaSuccess) {
            rc = QLD_ERR_CUDA; break;
        }
        for (int i = 0; i < 2; ++i)
            if (cudaEventCreateWithFlags(&c->ev_band[i], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->ev_copy[i], cudaEventDisableTiming) != cudaSuccess) {
                rc = QLD_ERR_CUDA; break;
            }
        if (rc) break;
        if (cudaMalloc(&c->d_status, sizeof(unsigned)) != cudaSuccess ||
            cudaMemset(c->d_status, 0, sizeof(unsigned)) != cudaSuccess ||
            cudaMallocHost(&c->h_status, sizeof(unsigned)) != cudaSuccess) {
            rc = QLD_ERR_NOMEM; break;
        }
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
                cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
            rc = QLD_ERR_CUDA; break;
        }
        c->encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    } while (0);
    if (rc) {
        cudaGetLastError();
        qld_cuda_release(c);
        return rc;
    }
    *ctx_out = c;
    return QLD_OK;
}

int qld_cuda_release(qld_ctx *c) {
    if (!c) return QLD_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy) cudaStreamSynchronize(c->copy);
    if (c->h2d) cudaStreamSynchronize(c->h2d);
    for (qld_batch_plan *p : c->plans) destroy_plan(p);
    c->plans.clear();
    for (cudaEvent_t e : c->h2d_ev) cudaEventDestroy(e);
    DevBuf *bufs[] = {&c->dA,       &c->dB,       &c->dbcA,     &c->dbcB,     &c->dOut[0],
                      &c->dOut[1],  &c->dCnt[0],  &c->dCnt[1],  &c->dJobs,    &c->dQueue,
                      &c->dMask[0], &c->dMask[1], &c->dHcnt[0], &c->dHcnt[1], &c->dHoff[0],
                      &c->dHoff[1], &c->dHval[0], &c->dHval[1], &c->vText,    &c->vSites,
                      &c->vValid,   &c->vSlash,   &c->vRoff,    &c->vRnd,     &c->vScratch,
                      &c->vWords,   &c->vBc,      &c->vLen,     &c->vKeep,    &c->vErr,
                      &c->dStage};
    for (DevBuf *b : bufs)
        if (b->p) cudaFree(b->p);
    HostBuf *hbufs[] = {&c->hMask[0], &c->hMask[1], &c->hOff[0], &c->hOff[1],
                        &c->hVal[0],  &c->hVal[1],  &c->hStat};
    for (HostBuf *b : hbufs)
        if (b->p) cudaFreeHost(b->p);
    for (auto &e : c->prof) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    for (int i = 0; i < 2; ++i) {
        if (c->ev_band[i]) cudaEventDestroy(c->ev_band[i]);
        if (c->ev_copy[i]) cudaEventDestroy(c->ev_copy[i]);
    }
    if (c->d_status) cudaFree(c->d_status);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->copy) cudaStreamDestroy(c->copy);
    if (c->h2d) cudaStreamDestroy(c->h2d);
    delete c;
    return QLD_OK;
}

const char *qld_cuda_last_error(const qld_ctx *c) { return c ? c->err : "no context"; }

int qld_cuda_set_option(qld_ctx *c, int option, long long value) {
    if (!c) return QLD_ERR_INVALID;
    switch (option) {
    case QLD_OPT_KERNEL:
        if (value < QLD_KERNEL_AUTO || value > QLD_KERNEL_FP4)
            return set_err(c, QLD_ERR_INVALID, "bad kernel variant %lld", value);
        c->kernel = (int)value;
        return QLD_OK;
    case QLD_OPT_R2_MODE:
        if (value != QLD_R2_EXACT && value != QLD_R2_REFERENCE)
            return set_err(c, QLD_ERR_INVALID, "bad r2 mode %lld", value);
        c->r2_mode = (int)value;
        return QLD_OK;
    case QLD_OPT_PROFILE:
        c->profile = value ? 1 : 0;
        return QLD_OK;
    case QLD_OPT_MMA_TILE:
        if (value != 0 && value != 128 && value != 256)
            return set_err(c, QLD_ERR_INVALID, "MMA tile rows must be 0, 128 or 256");
        c->mma_tile = (int)value;
        return QLD_OK;
    case QLD_OPT_SM_PAIR:
        if (value < 0 || value > 2)
            return set_err(c, QLD_ERR_INVALID, "SMs per 4-bit tile must be 0, 1 or 2");
        c->sm_pair = (int)value;
        return QLD_OK;
    case QLD_OPT_MEM_CAP:
        if (value < 0) return set_err(c, QLD_ERR_INVALID, "memory cap %lld out of range", value);
        c->mem_cap = (size_t)value;
        return QLD_OK;
    case QLD_OPT_WAIT_CYCLES:
        if (value < 0)
            return set_err(c, QLD_ERR_INVALID, "wait budget %lld out of range", value);
        c->timeout_cycles = value ? value : 4000000000LL;
        return QLD_OK;
    case QLD_OPT_BAND_ROWS:
        if (value < 256 || value > (1 << 24))
            return set_err(c, QLD_ERR_INVALID, "band rows %lld out of range", value);
        c->band_rows = (int)((value + 255) / 256 * 256);
        return QLD_OK;
    default:
        return set_err(c, QLD_ERR_INVALID, "unknown option %d", option);
    }
}

int qld_cuda_get_stats(qld_ctx *c, qld_stats *out, int reset) {
    if (!c) return QLD_ERR_INVALID;
    if (out) *out = c->stats;
    if (reset) {
        const int last = c->stats.last_kernel;
        c->stats = qld_stats{};
        c->stats.last_kernel = last;
    }
    return QLD_OK;
}

int qld_cuda_host_alloc(qld_ctx *c, size_t bytes, void **ptr) {
    if (!c || !ptr) return QLD_ERR_INVALID;
    cudaSetDevice(c->device);
    if (cudaMallocHost(ptr, bytes ? bytes : 1) != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return set_err(c, QLD_ERR_NOMEM, "cudaMallocHost(%zu) failed", bytes);
    }
    return QLD_OK;
}

int qld_cuda_host_free(qld_ctx *c, void *ptr) {
    if (!c) return QLD_ERR_INVALID;
    if (ptr) CUDA_TRY(c, cudaFreeHost(ptr));
    return QLD_OK;
}

int qld_cuda_ld(qld_ctx *c, const uint64_t *A, const uint32_t *bcA, int m, const uint64_t *B,
                const uint32_t *bcB, int n, int K, int S, int symmetric, float *r2_out,
                uint32_t *counts_out) {
    if (!c) return QLD_ERR_INVALID;
    if (symmetric) { B = A; bcB = bcA; n = m; }
    if (m < 0 || n < 0 || K < 1 || S < 1)
        return set_err(c, QLD_ERR_INVALID, "bad sizes m=%d n=%d K=%d S=%d", m, n, K, S);
    if (m == 0 || n == 0) return QLD_OK;
    if (!A || !bcA || !B || !bcB || !r2_out)
        return set_err(c, QLD_ERR_INVALID, "NULL table, bit-count or output pointer");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const long long Kp = K + (K & 1);
    int rc;
    if ((rc = ensure(c, c->dA, (size_t)m * Kp * 8)) || (rc = ensure(c, c->dbcA, (size_t)m * 4)))
        return rc;
    if (!symmetric && ((rc = ensure(c, c->dB, (size_t)n * Kp * 8)) ||
                       (rc = ensure(c, c->dbcB, (size_t)n * 4))))
        return rc;
    uint64_t *dA = static_cast<uint64_t *>(c->dA.p);
    uint64_t *dB = symmetric ? dA : static_cast<uint64_t *>(c->dB.p);
    const uint32_t *dbcA = static_cast<const uint32_t *>(c->dbcA.p);
    const uint32_t *dbcB = symmetric ? dbcA : static_cast<const uint32_t *>(c->dbcB.p);
    const Task t{dA, dbcA, m, Kp, dB, dbcB, n, Kp, K, S, symmetric, 0};

    const int band = band_rows_for(c, t);   // whole tile rows of the task's kernel
    const int nbands = (n + band - 1) / band;
    const size_t slot_rows = (size_t)(n < band ? n : band);
    for (int s = 0; s < 2 && s < nbands; ++s) {
        if ((rc = ensure(c, c->dOut[s], slot_rows * m * 4))) return rc;
        if (counts_out && (rc = ensure(c, c->dCnt[s], slot_rows * m * 4))) return rc;
    }
    uint64_t *stage;
    if ((rc = ensure_stage(c, K, !symmetric && m > band ? m : band, &stage))) return rc;
    // Tables go up in chunks of `band` rows on the h2d stream, an event after
    // each, so each band's kernel starts once the rows it reads are resident
    // and the host->device copies overlap the device->host results.  A single
    // region runs its bands last to first: band [b0, b1) reads table rows
    // from b0 (less one A tile) to m, which the chunks uploaded last-first
    // provide early, and its small last bands start the result copies at once.
    while ((int)c->h2d_ev.size() < nbands) {
        cudaEvent_t e;
        CUDA_TRY(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->h2d_ev.push_back(e);
    }
    CUDA_TRY(c, cudaMemcpyAsync(c->dbcA.p, bcA, (size_t)m * 4, cudaMemcpyHostToDevice, c->h2d));
    if (!symmetric) {
        CUDA_TRY(c, cudaMemcpyAsync(c->dbcB.p, bcB, (size_t)n * 4, cudaMemcpyHostToDevice, c->h2d));
        if ((rc = upload_rows(c, dA, Kp, A, K, m, stage, c->h2d))) return rc;
    }
    for (int k = 0; k < nbands; ++k) {
        const int i = symmetric ? nbands - 1 - k : k;
        const int r0 = i * band, r1 = r0 + band < n ? r0 + band : n;
        if ((rc = upload_rows(c, dB + (size_t)r0 * Kp, Kp, B + (size_t)r0 * K, K, r1 - r0, stage,
                              c->h2d)))
            return rc;
        CUDA_TRY(c, cudaEventRecord(c->h2d_ev[i], c->h2d));
    }
    for (int k = 0; k < nbands; ++k) {
        const int bi = symmetric ? nbands - 1 - k : k;
        const int s = k & 1;
        const int b0 = bi * band, b1 = b0 + band < n ? b0 + band : n;
        // symmetric: the chunk holding row b0 - 256 (A tiles start at multiples
        // of 256), uploaded after every chunk above it
        const int need = symmetric ? (b0 >= 256 ? (b0 - 256) / band : 0) : bi;
        CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->h2d_ev[need], 0));
        if (k >= 2) CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->ev_copy[s], 0));
        float *r2s = static_cast<float *>(c->dOut[s].p);
        uint32_t *cs = counts_out ? static_cast<uint32_t *>(c->dCnt[s].p) : nullptr;
        if ((rc = launch_counts(c, t, b0, b1, r2s, m, cs, m, b0, c->stream))) return rc;
        CUDA_TRY(c, cudaEventRecord(c->ev_band[s], c->stream));
        CUDA_TRY(c, cudaStreamWaitEvent(c->copy, c->ev_band[s], 0));
        if (!symmetric) {
            CUDA_TRY(c, cudaMemcpyAsync(r2_out + (size_t)b0 * m, r2s, (size_t)(b1 - b0) * m * 4,
                                        cudaMemcpyDeviceToHost, c->copy));
            if (cs)
                CUDA_TRY(c, cudaMemcpyAsync(counts_out + (size_t)b0 * m, cs,
                                            (size_t)(b1 - b0) * m * 4, cudaMemcpyDeviceToHost,
                                            c->copy));
        } else {
            // Per 512 rows: columns [r0, m) hold every entry j >= i (fewer,
            // larger 2-D copies run closer to the link rate than per 128 rows).
            for (int r0 = b0; r0 < b1; r0 += 512) {
                const int r1 = r0 + 512 < b1 ? r0 + 512 : b1;
                const size_t w = (size_t)(m - r0) * 4;
                CUDA_TRY(c, cudaMemcpy2DAsync(r2_out + (size_t)r0 * m + r0, (size_t)m * 4,
                                              r2s + (size_t)(r0 - b0) * m + r0, (size_t)m * 4, w,
                                              r1 - r0, cudaMemcpyDeviceToHost, c->copy));
                if (cs)
                    CUDA_TRY(c, cudaMemcpy2DAsync(counts_out + (size_t)r0 * m + r0, (size_t)m * 4,
                                                  cs + (size_t)(r0 - b0) * m + r0, (size_t)m * 4,
                                                  w, r1 - r0, cudaMemcpyDeviceToHost, c->copy));
            }
        }
        CUDA_TRY(c, cudaEventRecord(c->ev_copy[s], c->copy));
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->copy));
    CUDA_TRY(c, cudaStreamSynchronize(c->h2d));
    return finish(c, c->stream);
}

int qld_cuda_ld_hits(qld_ctx *c, const uint64_t *A, const uint32_t *bcA, int m,
                     const uint64_t *B, const uint32_t *bcB, int n, int K, int S, int symmetric,
                     int triangle, float r2limit, qld_hits_fn fn, void *user) {
    if (!c) return QLD_ERR_INVALID;
    if (symmetric) { B = A; bcB = bcA; n = m; triangle = 1; }
    if (m < 0 || n < 0 || K < 1 || S < 1)
        return set_err(c, QLD_ERR_INVALID, "bad sizes m=%d n=%d K=%d S=%d", m, n, K, S);
    if (!fn) return set_err(c, QLD_ERR_INVALID, "NULL block callback");
    if (m == 0 || n == 0) return QLD_OK;
    if (!A || !bcA || !B || !bcB)
        return set_err(c, QLD_ERR_INVALID, "NULL table or bit-count pointer");
    CUDA_TRY(c, cudaSetDevice(c->device));
    Task t;
    int rc;
    if ((rc = stage_tables(c, A, bcA, m, B, bcB, n, K, S, symmetric, &t))) return rc;

    const int BR = band_rows_for(c, t);      // whole tile rows of the task's kernel
    const int rows_blk = n < BR ? n : BR;
    const int nblk = (n + BR - 1) / BR;
    const long long ldr = ((long long)m + 127) / 128 * 128;   // float4 groups of 128 columns
    const int W = (m + 31) / 32;
    for (int s = 0; s < 2 && s < nblk; ++s) {
        if ((rc = ensure(c, c->dOut[s], (size_t)rows_blk * ldr * 4)) ||
            (rc = ensure(c, c->dMask[s], (size_t)rows_blk * W * 4)) ||
            (rc = ensure(c, c->dHcnt[s], (size_t)rows_blk * 8)) ||
            (rc = ensure(c, c->dHoff[s], (size_t)(rows_blk + 1) * 8)) ||
            (rc = ensure(c, c->dHval[s], (size_t)rows_blk * m * 4)) ||
            (rc = ensure_host(c, c->hMask[s], (size_t)rows_blk * W * 4)) ||
            (rc = ensure_host(c, c->hOff[s], (size_t)(rows_blk + 1) * 8)))
            return rc;
    }
    if ((rc = ensure_host(c, c->hStat, 2 * sizeof(unsigned)))) return rc;
    unsigned *hstat = static_cast<unsigned *>(c->hStat.p);

    // Block bi: counts + r^2 into dOut[s], the filter, then (copy stream)
    // the offsets, the mask and the status word to the host.
    auto issue = [&](int bi) -> int {
        const int s = bi & 1;
        const int b0 = bi * BR, b1 = b0 + BR < n ? b0 + BR : n;
        float *r2s = static_cast<float *>(c->dOut[s].p);
        int rc2;
        if ((rc2 = launch_counts(c, t, b0, b1, r2s, ldr, nullptr, 0, b0, c->stream))) return rc2;
        cudaError_t e = launch_hits(r2s, ldr, b1 - b0, m, b0, triangle, r2limit,
                                    static_cast<uint32_t *>(c->dMask[s].p),
                                    W, static_cast<long long *>(c->dHcnt[s].p),
                                    static_cast<long long *>(c->dHoff[s].p),
                                    static_cast<float *>(c->dHval[s].p), c->stream);
        if (e != cudaSuccess)
            return set_err(c, QLD_ERR_CUDA, "filter launch failed: %s", cudaGetErrorString(e));
        c->stats.kernel_launches += 3;
        CUDA_TRY(c, cudaEventRecord(c->ev_band[s], c->stream));
        CUDA_TRY(c, cudaStreamWaitEvent(c->copy, c->ev_band[s], 0));
        CUDA_TRY(c, cudaMemcpyAsync(c->hOff[s].p, c->dHoff[s].p, (size_t)(b1 - b0 + 1) * 8,
                                    cudaMemcpyDeviceToHost, c->copy));
        CUDA_TRY(c, cudaMemcpyAsync(c->hMask[s].p, c->dMask[s].p, (size_t)(b1 - b0) * W * 4,
                                    cudaMemcpyDeviceToHost, c->copy));
        CUDA_TRY(c, cudaMemcpyAsync(hstat + s, c->d_status, sizeof(unsigned),
                                    cudaMemcpyDeviceToHost, c->copy));
        CUDA_TRY(c, cudaEventRecord(c->ev_copy[s], c->copy));
        return QLD_OK;
    };
    // Wait for block bi's offsets and mask, fetch its values, call fn.
    auto consume = [&](int bi) -> int {
        const int s = bi & 1;
        const int b0 = bi * BR, b1 = b0 + BR < n ? b0 + BR : n;
        CUDA_TRY(c, cudaEventSynchronize(c->ev_copy[s]));
        if (hstat[s]) return QLD_ERR_TIMEOUT;
        const long long *off = static_cast<const long long *>(c->hOff[s].p);
        const long long total = off[b1 - b0];
        int rc2;
        if ((rc2 = ensure_host(c, c->hVal[s], (size_t)(total > 0 ? total : 1) * 4))) return rc2;
        if (total > 0) {
            CUDA_TRY(c, cudaMemcpyAsync(c->hVal[s].p, c->dHval[s].p, (size_t)total * 4,
                                        cudaMemcpyDeviceToHost, c->copy));
            CUDA_TRY(c, cudaStreamSynchronize(c->copy));
        }
        qld_hits_block blk;
        blk.row0 = b0;
        blk.rows = b1 - b0;
        blk.m = m;
        blk.words = W;
        blk.mask = static_cast<const uint32_t *>(c->hMask[s].p);
        blk.row_off = off;
        blk.val = static_cast<const float *>(c->hVal[s].p);
        c->stats.hits_rows += blk.rows;
        c->stats.hits_pairs += total;
        return fn(user, &blk);
    };
    rc = issue(0);
    for (int bi = 1; rc == QLD_OK && bi <= nblk; ++bi) {
        if (bi < nblk && (rc = issue(bi))) break;
        rc = consume(bi - 1);
    }
    // Drain whatever is still queued, then report a kernel that gave up.
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(c->copy);
    const int frc = finish(c, c->stream);
    if (rc == QLD_ERR_TIMEOUT || (rc == QLD_OK && frc != QLD_OK))
        return frc != QLD_OK ? frc
                             : set_err(c, QLD_ERR_TIMEOUT, "a counts kernel gave up a bounded wait");
    return rc;
}

int qld_cuda_count_states(qld_ctx *c, const uint64_t *A, int m, const uint64_t *B, int n, int K,
                          int symmetric, uint8_t *states_out) {
    if (!c) return QLD_ERR_INVALID;
    if (symmetric) { B = A; n = m; }
    if (m < 0 || n < 0 || K < 1)
        return set_err(c, QLD_ERR_INVALID, "bad sizes m=%d n=%d K=%d", m, n, K);
    if (m == 0 || n == 0) return QLD_OK;
    if (!A || !B || !states_out)
        return set_err(c, QLD_ERR_INVALID, "NULL table or output pointer");
    CUDA_TRY(c, cudaSetDevice(c->device));
    Task t;
    int rc;
    if ((rc = stage_tables(c, A, nullptr, m, B, nullptr, n, K, 1, symmetric, &t))) return rc;
    const int band = c->band_rows;
    const int nbands = (n + band - 1) / band;
    const size_t slot_rows = (size_t)(n < band ? n : band);
    for (int s = 0; s < 2 && s < nbands; ++s)
        if ((rc = ensure(c, c->dOut[s], slot_rows * m))) return rc;
    for (int bi = 0; bi < nbands; ++bi) {
        const int s = bi & 1;
        const int b0 = bi * band, b1 = b0 + band < n ? b0 + band : n;
        if (bi >= 2) CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->ev_copy[s], 0));
        uint8_t *os = static_cast<uint8_t *>(c->dOut[s].p);
        if ((rc = launch_states_range(c, t, b0, b1, os, m, b0, c->stream))) return rc;
        CUDA_TRY(c, cudaEventRecord(c->ev_band[s], c->stream));
        CUDA_TRY(c, cudaStreamWaitEvent(c->copy, c->ev_band[s], 0));
        CUDA_TRY(c, cudaMemcpyAsync(states_out + (size_t)b0 * m, os, (size_t)(b1 - b0) * m,
                                    cudaMemcpyDeviceToHost, c->copy));
        CUDA_TRY(c, cudaEventRecord(c->ev_copy[s], c->copy));
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->copy));
    return finish(c, c->stream);
}

int qld_cuda_count_states_device(qld_ctx *c, const uint64_t *A, int m, long long lda,
                                 const uint64_t *B, int n, long long ldb, int K, int symmetric,
                                 uint8_t *states, long long lds, void *stream) {
    if (!c) return QLD_ERR_INVALID;
    if (symmetric) { B = A; n = m; ldb = lda; }
    if (m < 0 || n < 0 || K < 1 || lda < K || ldb < K || (lda & 1) || (ldb & 1) || lds < m)
        return set_err(c, QLD_ERR_INVALID, "bad sizes/strides m=%d n=%d K=%d lda=%lld ldb=%lld",
                       m, n, K, lda, ldb);
    if (m == 0 || n == 0) return QLD_OK;
    if (!A || !B || !states || !aligned16(A) || !aligned16(B))
        return set_err(c, QLD_ERR_INVALID, "NULL or misaligned device pointer");
    CUDA_TRY(c, cudaSetDevice(c->device));
    Task t{A, nullptr, m, lda, B, nullptr, n, ldb, K, 1, symmetric, 0};
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    return launch_states_range(c, t, 0, n, states, lds, 0, st);
}

int qld_cuda_vcf_pack(qld_ctx *c, const char *text, size_t text_bytes,
                      const qld_vcf_site *sites, int nsites, const uint8_t *valid, int nsamples,
                      int ploidy, int K, qld_rand_fn rng, void *rng_user, uint64_t *words,
                      uint32_t *bc, int *snip_len, uint8_t *keep, int *err_site) {
    if (!c) return QLD_ERR_INVALID;
    if (err_site) *err_site = -1;
    if (nsites < 0 || nsamples < 1 || ploidy < 1 || K < 1 || (long long)K * 64 > (1LL << 30))
        return set_err(c, QLD_ERR_INVALID, "bad sizes nsites=%d nsamples=%d ploidy=%d K=%d",
                       nsites, nsamples, ploidy, K);
    if (nsites == 0) return QLD_OK;
    if (!text || !sites || !valid || !words || !bc || !snip_len || !keep)
        return set_err(c, QLD_ERR_INVALID, "NULL argument");
    for (int i = 0; i < nsites; ++i) {
        const qld_vcf_site &v = sites[i];
        if (v.off < 0 || v.len < 0 || (unsigned long long)v.off + (unsigned)v.len > text_bytes ||
            v.gt_pos < 0 || v.n_states < 0 || v.n_states > 4)
            return set_err(c, QLD_ERR_INVALID, "site %d lies outside the text or is malformed", i);
    }
    CUDA_TRY(c, cudaSetDevice(c->device));
    const int ctas = nsites < c->sm_count * 8 ? nsites : c->sm_count * 8;
    const int scratch_cap = K * 64;
    const size_t ns = (size_t)nsites;
    int rc;
    if ((rc = ensure(c, c->vText, text_bytes ? text_bytes : 1)) ||
        (rc = ensure(c, c->vSites, ns * sizeof(qld_vcf_site))) ||
        (rc = ensure(c, c->vValid, (size_t)nsamples)) || (rc = ensure(c, c->vSlash, ns * 8)) ||
        (rc = ensure(c, c->vRoff, ns * 8)) ||
        (rc = ensure(c, c->vScratch, (size_t)ctas * scratch_cap)) ||
        (rc = ensure(c, c->vWords, ns * K * 8)) || (rc = ensure(c, c->vBc, ns * 4)) ||
        (rc = ensure(c, c->vLen, ns * 4)) || (rc = ensure(c, c->vKeep, ns)) ||
        (rc = ensure(c, c->vErr, ns * 4)))
        return rc;
    cudaStream_t st = c->stream;
    CUDA_TRY(c, cudaMemcpyAsync(c->vText.p, text, text_bytes, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(c->vSites.p, sites, ns * sizeof(qld_vcf_site),
                                cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(c->vValid.p, valid, (size_t)nsamples, cudaMemcpyHostToDevice, st));
    const char *dtext = static_cast<const char *>(c->vText.p);
    const qld_vcf_site *dsites = static_cast<const qld_vcf_site *>(c->vSites.p);
    const uint8_t *dvalid = static_cast<const uint8_t *>(c->vValid.p);
    // 1. count: random draws per site
    cudaError_t e = launch_vcf_sites(dtext, dsites, nsites, dvalid, nsamples, ploidy, K, nullptr,
                                     nullptr, static_cast<long long *>(c->vSlash.p),
                                     static_cast<char *>(c->vScratch.p), scratch_cap, ctas,
                                     static_cast<uint64_t *>(c->vWords.p),
                                     static_cast<uint32_t *>(c->vBc.p),
                                     static_cast<int *>(c->vLen.p),
                                     static_cast<uint8_t *>(c->vKeep.p),
                                     static_cast<int *>(c->vErr.p), st);
    if (e != cudaSuccess)
        return set_err(c, QLD_ERR_CUDA, "VCF count launch failed: %s", cudaGetErrorString(e));
    std::vector<long long> slash(ns), roff(ns);
    CUDA_TRY(c, cudaMemcpyAsync(slash.data(), c->vSlash.p, ns * 8, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    long long total = 0;
    for (size_t i = 0; i < ns; ++i) {
        roff[i] = total;
        total += slash[i] > 0 ? slash[i] : 0;
    }
    if (total > 0 && !rng)
        return set_err(c, QLD_ERR_INVALID,
                       "unphased genotypes need %lld random draws and no generator was given",
                       total);
    std::vector<unsigned> rnd((size_t)(total > 0 ? total : 1));
    for (long long i = 0; i < total; ++i) rnd[(size_t)i] = rng(rng_user);
    if ((rc = ensure(c, c->vRnd, rnd.size() * 4))) return rc;
    CUDA_TRY(c, cudaMemcpyAsync(c->vRnd.p, rnd.data(), rnd.size() * 4, cudaMemcpyHostToDevice, st));
    CUDA_TRY(c, cudaMemcpyAsync(c->vRoff.p, roff.data(), ns * 8, cudaMemcpyHostToDevice, st));
    // 2. pack
    e = launch_vcf_sites(dtext, dsites, nsites, dvalid, nsamples, ploidy, K,
                         static_cast<const unsigned *>(c->vRnd.p),
                         static_cast<const long long *>(c->vRoff.p),
                         static_cast<long long *>(c->vSlash.p), static_cast<char *>(c->vScratch.p),
                         scratch_cap, ctas, static_cast<uint64_t *>(c->vWords.p),
                         static_cast<uint32_t *>(c->vBc.p), static_cast<int *>(c->vLen.p),
                         static_cast<uint8_t *>(c->vKeep.p), static_cast<int *>(c->vErr.p), st);
    if (e != cudaSuccess)
        return set_err(c, QLD_ERR_CUDA, "VCF pack launch failed: %s", cudaGetErrorString(e));
    c->stats.kernel_launches += 2;
    std::vector<int> err(ns);
    CUDA_TRY(c, cudaMemcpyAsync(words, c->vWords.p, ns * K * 8, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaMemcpyAsync(bc, c->vBc.p, ns * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaMemcpyAsync(snip_len, c->vLen.p, ns * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaMemcpyAsync(keep, c->vKeep.p, ns, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaMemcpyAsync(err.data(), c->vErr.p, ns * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(c, cudaStreamSynchronize(st));
    static const char *const what[] = {"",
                                       "empty GT field",
                                       "allele index past the REF/ALT states",
                                       "more than three alleles in a genotype",
                                       "more sample fields than header samples",
                                       "Detected data bigger than the ploidy of input",
                                       "a genotype with fewer alleles than separators",
                                       "no alleles (empty alignment)",
                                       "a state character qLD cannot map"};
    for (int i = 0; i < nsites; ++i) {
        const int code = err[(size_t)i];
        if (!code) continue;
        if (err_site) *err_site = i;
        return set_err(c, QLD_ERR_INVALID, "site %d: %s", i,
                       code > 0 && code <= 8 ? what[code] : "error");
    }
    return QLD_OK;
}

int qld_cuda_ld_device(qld_ctx *c, const qld_ld_args *a, void *stream) {
    if (!c || !a) return QLD_ERR_INVALID;
    Task t{a->A, a->bcA, a->m, a->lda, a->B, a->bcB, a->n, a->ldb, a->K, a->S, a->symmetric, 0};
    if (t.symmetric) { t.B = t.A; t.bcB = t.bcA; t.n = t.m; t.ldb = t.lda; }
    if (t.m < 0 || t.n < 0 || t.K < 1 || t.S < 1 || t.lda < t.K || t.ldb < t.K || (t.lda & 1) ||
        (t.ldb & 1) || a->ldr < t.m || (a->counts && a->ldc < t.m))
        return set_err(c, QLD_ERR_INVALID, "bad sizes/strides m=%d n=%d K=%d lda=%lld ldb=%lld",
                       t.m, t.n, t.K, t.lda, t.ldb);
    if (t.m == 0 || t.n == 0) return QLD_OK;
    if (!t.A || !t.B || !t.bcA || !t.bcB || !a->r2 || !aligned16(t.A) || !aligned16(t.B))
        return set_err(c, QLD_ERR_INVALID, "NULL or misaligned device pointer");
    CUDA_TRY(c, cudaSetDevice(c->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    return launch_counts(c, t, 0, t.n, a->r2, a->ldr, a->counts, a->ldc, 0, st);
}

int qld_cuda_split_rows(int m, int n, int K, int symmetric, int kernel, int part, int nparts,
                        int *row0, int *row1) {
    if (symmetric) n = m;
    if (m < 0 || n < 0 || K < 1 || nparts < 1 || part < 0 || part >= nparts || !row0 || !row1)
        return QLD_ERR_INVALID;
    Task t{nullptr, nullptr, m, K + (K & 1), nullptr, nullptr, n, K + (K & 1), K, 64 * K,
           symmetric, 0};
    if (kernel == QLD_KERNEL_AUTO) kernel = fp4_exact_for(t) ? QLD_KERNEL_FP4 : QLD_KERNEL_POPC;
    if (kernel != QLD_KERNEL_POPC && kernel != QLD_KERNEL_MMA && kernel != QLD_KERNEL_FP4)
        return QLD_ERR_INVALID;
    const KernelShape &ks = split_shape(kernel);
    split_rows(t, ks.bm, ks.bn, part, nparts, row0, row1);
    return QLD_OK;
}

int qld_cuda_ld_device_part(qld_ctx *c, const qld_ld_args *a, int part, int nparts, int *row0,
                            int *row1, void *stream) {
    if (!c || !a || !row0 || !row1 || nparts < 1 || part < 0 || part >= nparts)
        return QLD_ERR_INVALID;
    Task t{a->A, a->bcA, a->m, a->lda, a->B, a->bcB, a->n, a->ldb, a->K, a->S, a->symmetric, 0};
    if (t.symmetric) { t.B = t.A; t.bcB = t.bcA; t.n = t.m; t.ldb = t.lda; }
    if (t.m < 0 || t.n < 0 || t.K < 1 || t.S < 1 || t.lda < t.K || t.ldb < t.K || (t.lda & 1) ||
        (t.ldb & 1) || a->ldr < t.m || (a->counts && a->ldc < t.m))
        return set_err(c, QLD_ERR_INVALID, "bad sizes/strides m=%d n=%d K=%d lda=%lld ldb=%lld",
                       t.m, t.n, t.K, t.lda, t.ldb);
    const int variant = variant_of(c, t);
    const KernelShape &ks = shape_of(c, variant, t, 0, t.n);
    split_rows(t, ks.bm, ks.bn, part, nparts, row0, row1);
    if (t.m == 0 || *row0 >= *row1) return QLD_OK;
    if (!t.A || !t.B || !t.bcA || !t.bcB || !a->r2 || !aligned16(t.A) || !aligned16(t.B))
        return set_err(c, QLD_ERR_INVALID, "NULL or misaligned device pointer");
    CUDA_TRY(c, cudaSetDevice(c->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    return launch_counts(c, t, *row0, *row1, a->r2, a->ldr, a->counts, a->ldc, *row0, st);
}

int qld_cuda_ld_band_device(qld_ctx *c, const uint64_t *A, const uint32_t *bcA, int m,
                            long long lda, int K, int S, int band, float *r2_band, long long ldr,
                            uint32_t *counts_band, long long ldc, void *stream) {
    if (!c) return QLD_ERR_INVALID;
    if (m < 0 || K < 1 || S < 1 || band < 1 || lda < K || (lda & 1) || ldr < band ||
        (counts_band && ldc < band))
        return set_err(c, QLD_ERR_INVALID, "bad band sizes m=%d K=%d band=%d lda=%lld ldr=%lld", m,
                       K, band, lda, ldr);
    if (m == 0) return QLD_OK;
    if (!A || !bcA || !r2_band || !aligned16(A))
        return set_err(c, QLD_ERR_INVALID, "NULL or misaligned device pointer");
    CUDA_TRY(c, cudaSetDevice(c->device));
    Task t{A, bcA, m, lda, A, bcA, m, lda, K, S, 1, band};
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    return launch_counts(c, t, 0, m, r2_band, ldr, counts_band, ldc, 0, st);
}

int qld_cuda_ld_band(qld_ctx *c, const uint64_t *A, const uint32_t *bcA, int m, int K, int S,
                     int band, float *r2_band, uint32_t *counts_band) {
    if (!c) return QLD_ERR_INVALID;
    if (m < 0 || K < 1 || S < 1 || band < 1)
        return set_err(c, QLD_ERR_INVALID, "bad band sizes m=%d K=%d S=%d band=%d", m, K, S, band);
    if (m == 0) return QLD_OK;
    if (!A || !bcA || !r2_band)
        return set_err(c, QLD_ERR_INVALID, "NULL table, bit-count or output pointer");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const long long Kp = K + (K & 1);
    int rc;
    if ((rc = ensure(c, c->dA, (size_t)m * Kp * 8)) || (rc = ensure(c, c->dbcA, (size_t)m * 4)))
        return rc;
    uint64_t *dA = static_cast<uint64_t *>(c->dA.p);
    Task t{dA, static_cast<const uint32_t *>(c->dbcA.p), m, Kp, dA,
           static_cast<const uint32_t *>(c->dbcA.p), m, Kp, K, S, 1, band};
    const int rows_blk = band_rows_for(c, t);                // whole tile rows of the kernel
    const int nblk = (m + rows_blk - 1) / rows_blk;
    for (int s = 0; s < 2 && s < nblk; ++s) {
        if ((rc = ensure(c, c->dOut[s], (size_t)rows_blk * band * 4))) return rc;
        if (counts_band && (rc = ensure(c, c->dCnt[s], (size_t)rows_blk * band * 4))) return rc;
    }
    uint64_t *stage;
    if ((rc = ensure_stage(c, K, rows_blk, &stage))) return rc;
    // Host->device in row chunks on the h2d stream, an event after each.
    while ((int)c->h2d_ev.size() < nblk) {
        cudaEvent_t e;
        CUDA_TRY(c, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->h2d_ev.push_back(e);
    }
    CUDA_TRY(c, cudaMemcpyAsync(c->dbcA.p, bcA, (size_t)m * 4, cudaMemcpyHostToDevice, c->h2d));
    for (int i = 0; i < nblk; ++i) {
        const int r0 = i * rows_blk, r1 = r0 + rows_blk < m ? r0 + rows_blk : m;
        if ((rc = upload_rows(c, dA + (size_t)r0 * Kp, Kp, A + (size_t)r0 * K, K, r1 - r0, stage,
                              c->h2d)))
            return rc;
        CUDA_TRY(c, cudaEventRecord(c->h2d_ev[i], c->h2d));
    }
    for (int bi = 0; bi < nblk; ++bi) {
        const int s = bi & 1;
        const int b0 = bi * rows_blk, b1 = b0 + rows_blk < m ? b0 + rows_blk : m;
        // Rows a kernel on B rows [b0, b1) can touch: up to b1 + band plus a tile.
        const long long need = (long long)b1 + band + 512;
        const int last_chunk = (int)(((need < m ? need : m) - 1) / rows_blk);
        CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->h2d_ev[last_chunk], 0));
        if (bi >= 2) CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->ev_copy[s], 0));
        float *r2s = static_cast<float *>(c->dOut[s].p);
        uint32_t *cs = counts_band ? static_cast<uint32_t *>(c->dCnt[s].p) : nullptr;
        if ((rc = launch_counts(c, t, b0, b1, r2s, band, cs, band, b0, c->stream))) return rc;
        CUDA_TRY(c, cudaEventRecord(c->ev_band[s], c->stream));
        CUDA_TRY(c, cudaStreamWaitEvent(c->copy, c->ev_band[s], 0));
        CUDA_TRY(c, cudaMemcpyAsync(r2_band + (size_t)b0 * band, r2s, (size_t)(b1 - b0) * band * 4,
                                    cudaMemcpyDeviceToHost, c->copy));
        if (cs)
            CUDA_TRY(c, cudaMemcpyAsync(counts_band + (size_t)b0 * band, cs,
                                        (size_t)(b1 - b0) * band * 4, cudaMemcpyDeviceToHost,
                                        c->copy));
        CUDA_TRY(c, cudaEventRecord(c->ev_copy[s], c->copy));
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->copy));
    CUDA_TRY(c, cudaStreamSynchronize(c->h2d));
    return finish(c, c->stream);
}

// Per-job kernel choice: a job goes into the persistent launch when its
// kernel (variant_of: the context's forced kernel, else the autotuner's entry
// for its shape class, else the built-in rule) is the 4-bit one, and runs as
// its own launch of the chosen kernel after it otherwise (the popcount
// kernel past 2^24 samples, or a class the tuner found faster elsewhere).
int qld_cuda_ld_batch(qld_ctx *c, const qld_ld_args *jobs, int njobs, void *stream) {
    if (!c || (njobs > 0 && !jobs) || njobs < 0) return QLD_ERR_INVALID;
    if (njobs == 0) return QLD_OK;
    CUDA_TRY(c, cudaSetDevice(c->device));
    std::vector<RoutedTask> routed;
    long long items = 0;
    int rc;
    if ((rc = prepare_batch(c, jobs, njobs, c->hJobs, routed, items))) return rc;
    const int nb = (int)c->hJobs.size();
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    if (items > 0) {
        if ((rc = ensure(c, c->dJobs, sizeof(BatchJob) * (size_t)nb)) ||
            (rc = ensure(c, c->dQueue, sizeof(unsigned long long))))
            return rc;
        CUDA_TRY(c, cudaMemcpyAsync(c->dJobs.p, c->hJobs.data(), sizeof(BatchJob) * (size_t)nb,
                                    cudaMemcpyHostToDevice, st));
    }
    return enqueue_batch(c, static_cast<const BatchJob *>(c->dJobs.p), nb, items,
                         static_cast<unsigned long long *>(c->dQueue.p), routed, st);
}

int qld_cuda_batch_plan(qld_ctx *c, const qld_ld_args *jobs, int njobs, qld_batch_plan **out) {
    if (!c || !out || (njobs > 0 && !jobs) || njobs < 0) return QLD_ERR_INVALID;
    *out = nullptr;
    CUDA_TRY(c, cudaSetDevice(c->device));
    std::vector<BatchJob> hj;
    std::vector<RoutedTask> routed;
    long long items = 0;
    int rc;
    if ((rc = prepare_batch(c, jobs, njobs, hj, routed, items))) return rc;
    qld_batch_plan *p = new (std::nothrow) qld_batch_plan();
    if (!p) return set_err(c, QLD_ERR_NOMEM, "batch plan: out of host memory");
    p->ctx = c;
    if ((rc = build_plan(c, p, hj, items, routed))) {
        destroy_plan(p);
        return rc;
    }
    c->plans.push_back(p);
    *out = p;
    return QLD_OK;
}

int qld_cuda_batch_run(qld_batch_plan *p, void *stream) {
    if (!p || !p->ctx) return QLD_ERR_INVALID;
    qld_ctx *c = p->ctx;
    CUDA_TRY(c, cudaSetDevice(c->device));
    if (!p->exec) return QLD_OK;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
    cudaEvent_t e1 = nullptr;
    int rc;
    if ((rc = prof_begin(c, st, &e1))) return rc;
    CUDA_TRY(c, cudaGraphLaunch(p->exec, st));
    if (e1) CUDA_TRY(c, cudaEventRecord(e1, st));
    CUDA_TRY(c, cudaEventRecord(p->done, st));
    c->stats.counts_launches += p->counts_launches;
    c->stats.kernel_launches += p->kernel_launches;
    c->stats.last_kernel = p->last_kernel;
    return QLD_OK;
}

int qld_cuda_batch_free(qld_batch_plan *p) {
    if (!p) return QLD_OK;
    qld_ctx *c = p->ctx;
    if (c) {
        c->plans.erase(std::remove(c->plans.begin(), c->plans.end(), p), c->plans.end());
        cudaSetDevice(c->device);
    }
    destroy_plan(p);
    return QLD_OK;
}

int qld_cuda_sync(qld_ctx *c, void *stream) {
    if (!c) return QLD_ERR_INVALID;
    CUDA_TRY(c, cudaSetDevice(c->device));
    return finish(c, stream ? static_cast<cudaStream_t>(stream) : c->stream);
}

int qld_cuda_autotune(qld_ctx *c, int m, int n, int K, int symmetric, int *kernel,
                      int *option, float *ms) {
    if (!c) return QLD_ERR_INVALID;
    if (symmetric) n = m;
    if (m < 1 || n < 1 || K < 1 || (long long)K * 64 > 0x7FFFFFFFLL)
        return set_err(c, QLD_ERR_INVALID, "bad tuning shape m=%d n=%d K=%d", m, n, K);
    CUDA_TRY(c, cudaSetDevice(c->device));
    const int mt = m < kTuneMaxSide ? m : kTuneMaxSide;
    const int nt = symmetric ? mt : (n < kTuneMaxSide ? n : kTuneMaxSide);
    const long long Kp = K + (K & 1);
    int rc;
    if ((rc = ensure(c, c->dA, (size_t)mt * Kp * 8)) || (rc = ensure(c, c->dbcA, (size_t)mt * 4)) ||
        (rc = ensure(c, c->dOut[0], (size_t)nt * mt * 4)))
        return rc;
    if (!symmetric && ((rc = ensure(c, c->dB, (size_t)nt * Kp * 8)) ||
                       (rc = ensure(c, c->dbcB, (size_t)nt * 4))))
        return rc;
    uint64_t *dA = static_cast<uint64_t *>(c->dA.p);
    uint64_t *dB = symmetric ? dA : static_cast<uint64_t *>(c->dB.p);
    uint32_t *dbcA = static_cast<uint32_t *>(c->dbcA.p);
    uint32_t *dbcB = symmetric ? dbcA : static_cast<uint32_t *>(c->dbcB.p);
    k_tune_fill<<<1024, 256, 0, c->stream>>>(dA, mt, K, Kp, 0x5EEDull);
    k_tune_bc<<<(mt + 255) / 256, 256, 0, c->stream>>>(dA, mt, K, Kp, dbcA);
    if (!symmetric) {
        k_tune_fill<<<1024, 256, 0, c->stream>>>(dB, nt, K, Kp, 0xB0B0ull);
        k_tune_bc<<<(nt + 255) / 256, 256, 0, c->stream>>>(dB, nt, K, Kp, dbcB);
    }
    CUDA_TRY(c, cudaGetLastError());
    const Task t{dA, dbcA, mt, Kp, dB, dbcB, nt, Kp, K, K * 64, symmetric, 0};
    float *r2 = static_cast<float *>(c->dOut[0].p);

    struct Cand { int kernel, option; };
    std::vector<Cand> cands{{QLD_KERNEL_POPC, 0}};
    if (mma_exact_for(t)) { cands.push_back({QLD_KERNEL_MMA, 128}); cands.push_back({QLD_KERNEL_MMA, 256}); }
    if (fp4_exact_for(t)) { cands.push_back({QLD_KERNEL_FP4, 1}); cands.push_back({QLD_KERNEL_FP4, 2}); }

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUDA_TRY(c, cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return set_err(c, QLD_ERR_CUDA, "cudaEventCreate failed");
    }
    TuneChoice best{0, 0, 0.f};
    {
        OptionGuard guard(c);
        for (const Cand &cd : cands) {
            c->kernel = cd.kernel;
            c->mma_tile = cd.kernel == QLD_KERNEL_MMA ? cd.option : 0;
            c->sm_pair = cd.kernel == QLD_KERNEL_FP4 ? cd.option : 0;
            // one warm-up launch, then the mean of three
            if ((rc = launch_counts(c, t, 0, nt, r2, mt, nullptr, 0, 0, c->stream)) ||
                (rc = finish(c, c->stream)))
                break;
            cudaEventRecord(e0, c->stream);
            for (int r = 0; r < 3 && !rc; ++r)
                rc = launch_counts(c, t, 0, nt, r2, mt, nullptr, 0, 0, c->stream);
            cudaEventRecord(e1, c->stream);
            if (rc || (rc = finish(c, c->stream))) break;
            float el = 0.f;
            cudaEventElapsedTime(&el, e0, e1);
            if (best.kernel == 0 || el / 3 < best.ms) best = TuneChoice{cd.kernel, cd.option, el / 3};
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    c->tune[tune_key(m, n, K, (symmetric ? 1 : 0) + (c->r2_mode == QLD_R2_REFERENCE ? 4 : 0))] = best;
    if (kernel) *kernel = best.kernel;
    if (option) *option = best.option;
    if (ms) *ms = best.ms;
    return QLD_OK;
}

int qld_cuda_tune_save(qld_ctx *c, const char *path) {
    if (!c || !path) return QLD_ERR_INVALID;
    FILE *f = fopen(path, "w");
    if (!f) return set_err(c, QLD_ERR_INVALID, "cannot write %s", path);
    fprintf(f, "qld-tune 1\n");
    for (const auto &kv : c->tune)
        fprintf(f, "%d %d %d %d %d %d %.6f\n", (int)(kv.first >> 24), (int)((kv.first >> 16) & 255),
                (int)((kv.first >> 8) & 255), (int)(kv.first & 255), kv.second.kernel,
                kv.second.option, kv.second.ms);
    const bool ok = fclose(f) == 0;
    return ok ? QLD_OK : set_err(c, QLD_ERR_INVALID, "cannot write %s", path);
}

int qld_cuda_tune_load(qld_ctx *c, const char *path) {
    if (!c || !path) return QLD_ERR_INVALID;
    FILE *f = fopen(path, "r");
    if (!f) return set_err(c, QLD_ERR_INVALID, "cannot read %s", path);
    int version = 0;
    if (fscanf(f, "qld-tune %d", &version) != 1 || version != 1) {
        fclose(f);
        return set_err(c, QLD_ERR_INVALID, "%s is not a qld tuning table", path);
    }
    std::map<long long, TuneChoice> table;
    int ml, nl, kl, kind, kernel, option, line = 1;
    float ms;
    int got;
    while ((got = fscanf(f, "%d %d %d %d %d %d %f", &ml, &nl, &kl, &kind, &kernel, &option, &ms)) == 7) {
        ++line;
        const bool opt_ok = kernel == QLD_KERNEL_POPC ? option == 0
                            : kernel == QLD_KERNEL_MMA ? (option == 128 || option == 256)
                            : kernel == QLD_KERNEL_FP4 ? (option == 1 || option == 2)
                                                       : false;
        if (ml < 0 || ml > 31 || nl < 0 || nl > 31 || kl < 0 || kl > 31 ||
            (kind != 0 && kind != 1 && kind != 4 && kind != 5) ||
            !opt_ok || !(ms >= 0.f)) {
            fclose(f);
            return set_err(c, QLD_ERR_INVALID, "%s line %d: bad entry", path, line);
        }
        table[((long long)ml << 24) | ((long long)nl << 16) | ((long long)kl << 8) | kind] =
            TuneChoice{kernel, option, ms};
    }
    const bool at_end = got == EOF;
    fclose(f);
    if (!at_end) return set_err(c, QLD_ERR_INVALID, "%s line %d: bad entry", path, line + 1);
    for (const auto &kv : table) c->tune[kv.first] = kv.second;
    return QLD_OK;
}

}  // extern "C"
