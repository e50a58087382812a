// qld_serve.cu -- the serving loop (qld_srv_*, declared in include/qld_cuda.h).
//
// Tables live in HBM.  A worker thread owns all launches:
//   admission  pending queries, in arrival order, get their r^2 output from a
//              first-fit device pool while it has room (a query that does
//              not fit waits; later ones wait behind it);
//   batching   the admitted queries become the tasks of one persistent
//              batched launch (launch_batch, ld_batch.cu), whose epilogue
//              also folds each query's summary, on the first free stream
//              slot -- while the batches of earlier slots are still running;
//   completion a host function enqueued after each batch wakes the worker,
//              which publishes results, copies summaries out and returns pool
//              memory, so the next pending queries can be admitted.
#include <cudaTypedefs.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "qld_cuda.h"
#include "qld_kernels.h"
#include "tcgen05.cuh"

using namespace qld;

namespace {

constexpr int kMaxJobsPerBatch = 1024;

using Summary = BatchSummary;   // per query, folded by the batch kernel's epilogue

struct Table {
    uint64_t *d = nullptr;
    uint32_t *bc = nullptr;
    int m = 0, K = 0, S = 0;
    long long lda = 0;
};

enum QState { PENDING, RUNNING, DONE, RELEASED };

struct Query {
    long long id;
    qld_query q;
    std::chrono::steady_clock::time_point t_submit;
    size_t off = 0, bytes = 0;   // pool range of its r^2
    bool has_mem = false;
    QState state = PENDING;
    long long pairs = 0;
};

struct Slot {
    cudaStream_t st = nullptr;
    BatchJob *dJobs = nullptr, *hJobs = nullptr;
    Summary *dSum = nullptr, *hSum = nullptr;
    unsigned long long *dQueue = nullptr;
    unsigned *dStatus = nullptr, *hStatus = nullptr;
    std::vector<Query> qs;        // copies of the admitted queries (taken under the lock)
    bool busy = false;
    bool finished = false;        // set by the host function after the batch
    int launch_error = QLD_OK;
};

struct Pool {
    size_t size = 0;
    std::map<size_t, size_t> free_;   // offset -> length, coalesced
    size_t free_bytes = 0;
    void init(size_t n) { size = n; free_.clear(); free_[0] = n; free_bytes = n; }
    bool alloc(size_t n, size_t *off) {
        n = (n + 255) & ~size_t(255);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                *off = it->first;
                const size_t rest = it->second - n, o2 = it->first + n;
                free_.erase(it);
                if (rest) free_[o2] = rest;
                free_bytes -= n;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t n) {
        n = (n + 255) & ~size_t(255);
        free_bytes += n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

}  // namespace

struct qld_server {
    int device = 0;
    int sm_count = 0;
    char err[512] = {0};
    unsigned char *pool_base = nullptr;
    Pool pool;
    std::vector<Table> tables;
    std::vector<Slot> slots;
    std::unordered_map<long long, Query> queries;
    std::deque<long long> pending;
    std::deque<qld_query_result> done;
    long long next_id = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    std::thread worker;
    cudaStream_t fetch_st = nullptr;
    PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
};

namespace {

int srv_err(qld_server *s, int code, const char *fmt, ...) {
    if (s) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(s->err, sizeof s->err, fmt, ap);
        va_end(ap);
    }
    return code;
}

bool encode_map(qld_server *s, CUtensorMap *tm, const void *base, int rows, int K, long long ld,
                int box_rows) {
    const KernelShape &ks = kBatchShape;
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
    cuuint32_t box[2] = {(cuuint32_t)ks.box_words, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return s->encode(tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void *>(base), dims, strides,
                     box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void CUDART_CB batch_finished(void *arg) {
    // Runs on a driver thread: no CUDA calls here, only the hand-off.
    auto *pr = static_cast<std::pair<qld_server *, int> *>(arg);
    qld_server *s = pr->first;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->slots[pr->second].finished = true;
    }
    s->cv_work.notify_one();
    delete pr;
}

// Launch the admitted queries of slot `si` (worker thread, no lock held).
int launch_slot(qld_server *s, int si) {
    Slot &sl = s->slots[si];
    std::vector<Table> tables;   // add_table may grow the server's vector meanwhile
    {
        std::lock_guard<std::mutex> g(s->mu);
        tables = s->tables;
    }
    const int nj = (int)sl.qs.size();
    std::vector<int> order(nj);
    std::vector<long long> cost(nj), tiles(nj);
    for (int i = 0; i < nj; ++i) {
        const Query &q = sl.qs[i];
        const int m = q.q.a1 - q.q.a0, n = q.q.b1 - q.q.b0;
        const int sym = (q.q.a0 == q.q.b0 && q.q.a1 == q.q.b1);
        tiles[i] = tc::TileList<256, 240>{(m + 255) / 256, 0, (n + 239) / 240, sym, 0}.count();
        cost[i] = tiles[i] * (long long)tables[q.q.table].K;
        order[i] = i;
    }
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    long long items = 0;
    for (int k = 0; k < nj; ++k) {
        const int i = order[k];
        const Query &q = sl.qs[i];
        const Table &T = tables[q.q.table];
        const int m = q.q.a1 - q.q.a0, n = q.q.b1 - q.q.b0;
        const int sym = (q.q.a0 == q.q.b0 && q.q.a1 == q.q.b1);
        float *out = reinterpret_cast<float *>(s->pool_base + q.off);
        BatchJob &J = sl.hJobs[k];
        memset(&J, 0, sizeof J);
        const uint64_t *A = T.d + (size_t)q.q.a0 * T.lda, *B = T.d + (size_t)q.q.b0 * T.lda;
        if (!encode_map(s, &J.tmA, A, m, T.K, T.lda, kBatchShape.box_rows_a) ||
            !encode_map(s, &J.tmB, B, n, T.K, T.lda, kBatchShape.box_rows_b))
            return QLD_ERR_CUDA;
        J.bcA = T.bc + q.q.a0;
        J.bcB = T.bc + q.q.b0;
        J.r2 = out;
        J.ldr = m;
        J.item0 = items;
        J.m = m; J.n = n; J.K = T.K; J.S = T.S; J.symmetric = sym;
        J.threshold = q.q.threshold;
        J.summary = sl.dSum + i;
        items += tiles[i];
    }
    cudaStream_t st = sl.st;
    if (cudaMemcpyAsync(sl.dJobs, sl.hJobs, sizeof(BatchJob) * nj, cudaMemcpyHostToDevice, st) ||
        cudaMemsetAsync(sl.dQueue, 0, sizeof(unsigned long long), st) ||
        cudaMemsetAsync(sl.dStatus, 0, sizeof(unsigned), st) ||
        cudaMemsetAsync(sl.dSum, 0, sizeof(Summary) * nj, st))
        return QLD_ERR_CUDA;
    BatchParams bp{};
    bp.jobs = sl.dJobs;
    bp.njobs = nj;
    bp.nitems = items;
    bp.queue = sl.dQueue;
    bp.status = sl.dStatus;
    bp.timeout_cycles = 4000000000LL;
    if (items > 0 && launch_batch(bp, R2_EXACT, 0, st) != cudaSuccess) return QLD_ERR_CUDA;
    for (int i = 0; i < nj; ++i) {
        const Query &q = sl.qs[i];
        if (q.q.host_r2)
            if (cudaMemcpyAsync(q.q.host_r2, s->pool_base + q.off, q.bytes, cudaMemcpyDeviceToHost,
                                st))
                return QLD_ERR_CUDA;
    }
    if (cudaMemcpyAsync(sl.hSum, sl.dSum, sizeof(Summary) * nj, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(sl.hStatus, sl.dStatus, sizeof(unsigned), cudaMemcpyDeviceToHost, st))
        return QLD_ERR_CUDA;
    auto *arg = new std::pair<qld_server *, int>(s, si);
    if (cudaLaunchHostFunc(st, batch_finished, arg) != cudaSuccess) {
        delete arg;
        return QLD_ERR_CUDA;
    }
    return QLD_OK;
}

// Publish a finished slot (worker thread, lock held).
void complete_slot(qld_server *s, int si, int status) {
    Slot &sl = s->slots[si];
    const auto now = std::chrono::steady_clock::now();
    if (status == QLD_OK && *sl.hStatus) status = QLD_ERR_TIMEOUT;
    for (size_t i = 0; i < sl.qs.size(); ++i) {
        auto it = s->queries.find(sl.qs[i].id);
        if (it == s->queries.end()) continue;
        Query &q = it->second;
        qld_query_result r{};
        r.id = q.id;
        r.status = status;
        r.latency_ms = std::chrono::duration<double, std::milli>(now - q.t_submit).count();
        r.pairs = q.pairs;
        if (status == QLD_OK) {
            r.n_above = (long long)sl.hSum[i].n_above;
            r.sum_r2 = sl.hSum[i].sum;
            unsigned bits = sl.hSum[i].max_bits;
            memcpy(&r.max_r2, &bits, 4);
        }
        q.state = DONE;
        if ((q.q.host_r2 || status != QLD_OK) && q.has_mem) {
            s->pool.release(q.off, q.bytes);
            q.has_mem = false;
        }
        s->done.push_back(r);
    }
    sl.qs.clear();
    sl.busy = false;
    sl.finished = false;
}

void worker_main(qld_server *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progressed = false;
        for (size_t si = 0; si < s->slots.size(); ++si) {
            Slot &sl = s->slots[si];
            if (sl.busy && sl.finished) {
                lk.unlock();
                cudaStreamSynchronize(sl.st);   // the host function ran: the stream is idle
                lk.lock();
                complete_slot(s, (int)si, sl.launch_error);
                progressed = true;
            }
        }
        if (progressed) s->cv_done.notify_all();
        int busy = 0;
        for (auto &sl : s->slots) busy += sl.busy;
        if (s->stop && s->pending.empty() && busy == 0) break;
        int free_slot = -1;
        for (size_t si = 0; si < s->slots.size(); ++si)
            if (!s->slots[si].busy) { free_slot = (int)si; break; }
        if (free_slot >= 0 && !s->pending.empty()) {
            Slot &sl = s->slots[free_slot];
            // Admission: arrival order, while the pool has room.
            while (!s->pending.empty() && (int)sl.qs.size() < kMaxJobsPerBatch) {
                Query &q = s->queries.at(s->pending.front());
                if (!s->pool.alloc(q.bytes, &q.off)) break;
                q.has_mem = true;
                q.state = RUNNING;
                sl.qs.push_back(q);
                s->pending.pop_front();
            }
            if (!sl.qs.empty()) {
                sl.busy = true;
                sl.finished = false;
                lk.unlock();
                const int rc = launch_slot(s, free_slot);
                lk.lock();
                if (rc != QLD_OK) {
                    cudaGetLastError();
                    sl.launch_error = rc;
                    lk.unlock();
                    cudaStreamSynchronize(sl.st);
                    lk.lock();
                    complete_slot(s, free_slot, rc);
                    sl.launch_error = QLD_OK;
                    s->cv_done.notify_all();
                }
                continue;
            }
        }
        s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
    }
}

void free_slot_buffers(Slot &sl) {
    if (sl.st) cudaStreamSynchronize(sl.st);
    cudaFree(sl.dJobs); cudaFree(sl.dSum); cudaFree(sl.dQueue);
    cudaFree(sl.dStatus);
    cudaFreeHost(sl.hJobs); cudaFreeHost(sl.hSum);
    cudaFreeHost(sl.hStatus);
    if (sl.st) cudaStreamDestroy(sl.st);
}

}  // namespace

extern "C" {

int qld_srv_create(int device, size_t pool_bytes, int max_inflight, qld_server **out) {
    if (!out || pool_bytes == 0 || max_inflight < 1 || max_inflight > 16) return QLD_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return QLD_ERR_NODEVICE;
    }
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) return QLD_ERR_NODEVICE;
    qld_server *s = new (std::nothrow) qld_server();
    if (!s) return QLD_ERR_NOMEM;
    s->device = device;
    cudaSetDevice(device);
    cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device);
    int rc = QLD_OK;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) !=
            cudaSuccess || qr != cudaDriverEntryPointSuccess || !fn)
        rc = QLD_ERR_CUDA;
    s->encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    if (!rc && cudaMalloc(&s->pool_base, pool_bytes) != cudaSuccess) rc = QLD_ERR_NOMEM;
    if (!rc && cudaStreamCreateWithFlags(&s->fetch_st, cudaStreamNonBlocking) != cudaSuccess)
        rc = QLD_ERR_CUDA;
    s->slots.resize(max_inflight);
    for (auto &sl : s->slots) {
        if (rc) break;
        if (cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) ||
            cudaMalloc(&sl.dJobs, sizeof(BatchJob) * kMaxJobsPerBatch) ||
            cudaMalloc(&sl.dSum, sizeof(Summary) * kMaxJobsPerBatch) ||
            cudaMalloc(&sl.dQueue, sizeof(unsigned long long)) ||
            cudaMalloc(&sl.dStatus, sizeof(unsigned)) ||
            cudaMallocHost(&sl.hJobs, sizeof(BatchJob) * kMaxJobsPerBatch) ||
            cudaMallocHost(&sl.hSum, sizeof(Summary) * kMaxJobsPerBatch) ||
            cudaMallocHost(&sl.hStatus, sizeof(unsigned)))
            rc = QLD_ERR_NOMEM;
    }
    if (rc) {
        cudaGetLastError();
        for (auto &sl : s->slots) free_slot_buffers(sl);
        if (s->pool_base) cudaFree(s->pool_base);
        if (s->fetch_st) cudaStreamDestroy(s->fetch_st);
        delete s;
        return rc;
    }
    s->pool.init(pool_bytes);
    s->worker = std::thread(worker_main, s);
    *out = s;
    return QLD_OK;
}

const char *qld_srv_last_error(const qld_server *s) { return s ? s->err : "no server"; }

int qld_srv_add_table(qld_server *s, const uint64_t *A, const uint32_t *bc, int m, int K, int S,
                      int *table_id) {
    if (!s || !A || !bc || !table_id || m < 1 || K < 1 || S < 1)
        return srv_err(s, QLD_ERR_INVALID, "bad table arguments");
    if ((long long)K * 64 > kBatchMaxSamples)
        return srv_err(s, QLD_ERR_UNSUPPORTED, "K*64 > %d samples", kBatchMaxSamples);
    cudaSetDevice(s->device);
    Table T;
    T.m = m; T.K = K; T.S = S;
    T.lda = K + (K & 1);
    if (cudaMalloc(&T.d, (size_t)m * T.lda * 8) != cudaSuccess ||
        cudaMalloc(&T.bc, (size_t)m * 4) != cudaSuccess) {
        cudaGetLastError();
        if (T.d) cudaFree(T.d);
        return srv_err(s, QLD_ERR_NOMEM, "table of %d x %d words does not fit", m, K);
    }
    // cudaMemcpyDefault: the table may come from host or from device memory.
    // One 1-D copy, in place for even K, else into a staging buffer that a
    // kernel re-pitches (row-pitched 2-D copies from the host run at about a
    // third of the link rate); row by row only if the staging buffer does
    // not fit.
    const size_t bytes = (size_t)m * K * 8;
    bool ok = cudaMemcpy(T.bc, bc, (size_t)m * 4, cudaMemcpyDefault) == cudaSuccess;
    if (ok && T.lda == K) {
        ok = cudaMemcpy(T.d, A, bytes, cudaMemcpyDefault) == cudaSuccess;
    } else if (ok) {
        void *stage = nullptr;
        if (cudaMalloc(&stage, bytes) == cudaSuccess) {
            ok = cudaMemcpy(stage, A, bytes, cudaMemcpyDefault) == cudaSuccess &&
                 launch_pad_rows(T.d, T.lda, static_cast<const uint64_t *>(stage), K, m, 0) ==
                     cudaSuccess &&
                 cudaStreamSynchronize(0) == cudaSuccess;
            cudaFree(stage);
        } else {
            cudaGetLastError();
            ok = cudaMemcpy2D(T.d, T.lda * 8, A, (size_t)K * 8, (size_t)K * 8, m,
                              cudaMemcpyDefault) == cudaSuccess;
        }
    }
    if (!ok) {
        cudaGetLastError();
        cudaFree(T.d);
        cudaFree(T.bc);
        return srv_err(s, QLD_ERR_CUDA, "table upload failed");
    }
    std::lock_guard<std::mutex> g(s->mu);
    s->tables.push_back(T);
    *table_id = (int)s->tables.size() - 1;
    return QLD_OK;
}

int qld_srv_submit(qld_server *s, const qld_query *q, long long *id) {
    if (!s || !q || !id) return QLD_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) return srv_err(s, QLD_ERR_INVALID, "server is stopping");
    if (q->table < 0 || q->table >= (int)s->tables.size())
        return srv_err(s, QLD_ERR_INVALID, "unknown table %d", q->table);
    const Table &T = s->tables[q->table];
    if (q->a0 < 0 || q->a1 <= q->a0 || q->a1 > T.m || q->b0 < 0 || q->b1 <= q->b0 || q->b1 > T.m)
        return srv_err(s, QLD_ERR_INVALID, "query rows outside the table");
    if (q->host_r2) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, q->host_r2) != cudaSuccess ||
            at.type != cudaMemoryTypeHost) {
            cudaGetLastError();
            return srv_err(s, QLD_ERR_INVALID, "host_r2 must be pinned host memory");
        }
    }
    const long long m = q->a1 - q->a0, n = q->b1 - q->b0;
    Query Q;
    Q.id = s->next_id++;
    Q.q = *q;
    Q.t_submit = std::chrono::steady_clock::now();
    Q.bytes = (size_t)m * (size_t)n * 4;
    Q.pairs = (q->a0 == q->b0 && q->a1 == q->b1) ? m * (m - 1) / 2 : m * n;
    if (Q.bytes > s->pool.size) {
        --s->next_id;
        return srv_err(s, QLD_ERR_BUSY, "query output %zu bytes exceeds the pool", Q.bytes);
    }
    s->queries.emplace(Q.id, Q);
    s->pending.push_back(Q.id);
    *id = Q.id;
    s->cv_work.notify_one();
    return QLD_OK;
}

int qld_srv_poll(qld_server *s, qld_query_result *out, int max, int *count, int wait_ms) {
    if (!s || !count || (max > 0 && !out)) return QLD_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms),
                            [&] { return !s->done.empty(); });
    int n = 0;
    while (n < max && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    *count = n;
    return QLD_OK;
}

int qld_srv_fetch(qld_server *s, long long id, float *host_r2) {
    if (!s || !host_r2) return QLD_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->queries.find(id);
    if (it == s->queries.end() || it->second.state != DONE || !it->second.has_mem)
        return srv_err(s, QLD_ERR_INVALID, "query %lld has no result on the device", id);
    const size_t off = it->second.off, bytes = it->second.bytes;
    lk.unlock();
    cudaSetDevice(s->device);
    if (cudaMemcpyAsync(host_r2, s->pool_base + off, bytes, cudaMemcpyDeviceToHost, s->fetch_st) !=
            cudaSuccess ||
        cudaStreamSynchronize(s->fetch_st) != cudaSuccess) {
        cudaGetLastError();
        return srv_err(s, QLD_ERR_CUDA, "fetch of query %lld failed", id);
    }
    return QLD_OK;
}

int qld_srv_release(qld_server *s, long long id) {
    if (!s) return QLD_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->queries.find(id);
    if (it == s->queries.end()) return srv_err(s, QLD_ERR_INVALID, "unknown query %lld", id);
    Query &q = it->second;
    if (q.state == RUNNING) return srv_err(s, QLD_ERR_BUSY, "query %lld is running", id);
    if (q.state == PENDING) {
        s->pending.erase(std::find(s->pending.begin(), s->pending.end(), id));
    } else if (q.has_mem) {
        s->pool.release(q.off, q.bytes);
    }
    s->queries.erase(it);
    s->cv_work.notify_one();
    return QLD_OK;
}

int qld_srv_destroy(qld_server *s) {
    if (!s) return QLD_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        // Pending queries are cancelled; running batches finish.
        for (long long id : s->pending) s->queries.erase(id);
        s->pending.clear();
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->device);
    for (auto &sl : s->slots) free_slot_buffers(sl);
    for (auto &T : s->tables) {
        cudaFree(T.d);
        cudaFree(T.bc);
    }
    if (s->pool_base) cudaFree(s->pool_base);
    if (s->fetch_st) cudaStreamDestroy(s->fetch_st);
    delete s;
    return QLD_OK;
}

}  // extern "C"
