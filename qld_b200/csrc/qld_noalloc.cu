// qld_noalloc.cu -- qld_cuda_ld_noalloc(): one LD task from host buffers
// without allocating any memory.
//
// Some callers cannot allocate device memory: a host program whose device
// memory is entirely reserved up front by another component (a pool or
// framework that owns the GPU's memory and forbids cudaMalloc/cudaFree
// outside it), or a plug-in loaded into such a program.  For them this entry
// point takes the same host tables and host result buffer as qld_cuda_ld()
// but creates no context, no stream, no event and no buffer: every device
// byte it needs -- the kernel status word, the staged tables and bit counts,
// and one r^2 output band -- lives in g_scratch, a file-scope static
// __device__ array of QLD_NOALLOC_SCRATCH_BYTES (16 MiB) that every GPU
// loading the library holds until the process exits.
//
// Host code never uses g_scratch directly: in host code that name is only a
// host-side stand-in, not a device address (a kernel given it would fault,
// or silently touch host memory where the GPU can reach it).  The first call
// on each device, with that device current, asks the runtime for the
// array's device address with cudaGetSymbolAddress() and caches it; do that
// first call before any stream capture.  All calls share the array and it
// keeps the previous call's contents (the status word is cleared at the
// start of every call); calls that overlap on the GPU -- on two streams, or
// from two threads -- race on it and must be serialized by the caller.
#include <cudaTypedefs.h>

#include <mutex>

#include "qld_cuda.h"
#include "qld_kernels.h"

using namespace qld;

namespace {

constexpr size_t kScratchBytes = QLD_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_lock;
unsigned char *g_scratch_dev[kMaxDevices];                 // device address per device
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Once per device, with the device current: the scratch array's device
// address, the device check, and the tensor-map encoder.
int setup(int dev, unsigned char **scratch) {
    if (dev < 0 || dev >= kMaxDevices) return QLD_ERR_NODEVICE;
    std::lock_guard<std::mutex> g(g_setup_lock);
    if (!g_scratch_dev[dev]) {
        int major = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) !=
                cudaSuccess ||
            major != 10) {
            cudaGetLastError();
            return QLD_ERR_NODEVICE;
        }
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return QLD_ERR_CUDA;
        }
        if (!g_encode) {
            void *fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
                    cudaSuccess ||
                q != cudaDriverEntryPointSuccess || !fn) {
                cudaGetLastError();
                return QLD_ERR_CUDA;
            }
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        }
        g_scratch_dev[dev] = static_cast<unsigned char *>(p);
    }
    *scratch = g_scratch_dev[dev];
    return QLD_OK;
}

bool make_map(CUtensorMap *tm, const void *base, int rows, int K, long long ld,
              const KernelShape &ks, bool is_a) {
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
    cuuint32_t box[2] = {(cuuint32_t)ks.box_words,
                         (cuuint32_t)(is_a ? ks.box_rows_a : ks.box_rows_b)};
    cuuint32_t estr[2] = {1, 1};
    const CUtensorMapSwizzle sw =
        ks.swizzle == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
    return g_encode(tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void *>(base), dims,
                    strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

#define NA_TRY(expr)                                  \
    do {                                              \
        if ((expr) != cudaSuccess) {                  \
            cudaGetLastError();                       \
            return QLD_ERR_CUDA;                      \
        }                                             \
    } while (0)

// Once work is queued on the caller's stream, a failure first waits for it:
// the copies still read the caller's host tables and write its r^2 buffer,
// and the next call must not find the shared scratch still in use.
#define NA_TRY_Q(expr)                                \
    do {                                              \
        if ((expr) != cudaSuccess) {                  \
            cudaGetLastError();                       \
            cudaStreamSynchronize(st);                \
            cudaGetLastError();                       \
            return QLD_ERR_CUDA;                      \
        }                                             \
    } while (0)

}  // namespace

extern "C" int qld_cuda_ld_noalloc(const uint64_t *A, const uint32_t *bcA, int m,
                                   const uint64_t *B, const uint32_t *bcB, int n, int K, int S,
                                   int symmetric, float *r2_out, void *stream) {
    if (symmetric) { B = A; bcB = bcA; n = m; }
    if (m < 0 || n < 0 || K < 1 || S < 1) return QLD_ERR_INVALID;
    if (m == 0 || n == 0) return QLD_OK;
    if (!A || !bcA || !B || !bcB || !r2_out) return QLD_ERR_INVALID;
    int dev = 0;
    NA_TRY(cudaGetDevice(&dev));
    unsigned char *scratch = nullptr;
    int rc = setup(dev, &scratch);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Scratch layout: status | bcA | bcB | A | B | r^2 band.
    const long long Kp = K + (K & 1);
    size_t off = 256;
    const size_t o_bcA = off;
    off = align256(off + (size_t)m * 4);
    const size_t o_bcB = off;
    if (!symmetric) off = align256(off + (size_t)n * 4);
    const size_t o_A = off;
    off = align256(off + (size_t)m * Kp * 8);
    const size_t o_B = off;
    if (!symmetric) off = align256(off + (size_t)n * Kp * 8);
    if (off >= kScratchBytes) return QLD_ERR_TOO_LARGE;
    const size_t o_band = off;
    const size_t band_rows_fit = (kScratchBytes - off) / ((size_t)m * 4);
    int band;
    if (band_rows_fit >= (size_t)n) band = n;
    else band = (int)(band_rows_fit / 256 * 256);   // whole 256-row tile rows
    if (band <= 0) return QLD_ERR_TOO_LARGE;

    unsigned *status = reinterpret_cast<unsigned *>(scratch);
    uint32_t *d_bcA = reinterpret_cast<uint32_t *>(scratch + o_bcA);
    uint32_t *d_bcB = symmetric ? d_bcA : reinterpret_cast<uint32_t *>(scratch + o_bcB);
    uint64_t *d_A = reinterpret_cast<uint64_t *>(scratch + o_A);
    uint64_t *d_B = symmetric ? d_A : reinterpret_cast<uint64_t *>(scratch + o_B);
    float *d_band = reinterpret_cast<float *>(scratch + o_band);

    // Each table goes up as one 1-D copy (row-pitched 2-D copies of a few KB
    // per row run at about a third of the link rate): in place for even K,
    // else through the r^2 band area (unused until the first kernel) and a
    // padding kernel; row by row only when the band area cannot hold it.
    auto upload = [&](uint64_t *dst, const uint64_t *src, int rows) -> int {
        const size_t bytes = (size_t)rows * K * 8;
        if (Kp == K) {
            NA_TRY_Q(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
        } else if (bytes <= kScratchBytes - o_band) {
            uint64_t *stage = reinterpret_cast<uint64_t *>(scratch + o_band);
            NA_TRY_Q(cudaMemcpyAsync(stage, src, bytes, cudaMemcpyHostToDevice, st));
            NA_TRY_Q(launch_pad_rows(dst, Kp, stage, K, rows, st));
        } else {
            NA_TRY_Q(cudaMemcpy2DAsync(dst, Kp * 8, src, (size_t)K * 8, (size_t)K * 8, rows,
                                     cudaMemcpyHostToDevice, st));
        }
        return QLD_OK;
    };
    NA_TRY_Q(cudaMemsetAsync(status, 0, sizeof(unsigned), st));
    if ((rc = upload(d_A, A, m))) return rc;
    NA_TRY_Q(cudaMemcpyAsync(d_bcA, bcA, (size_t)m * 4, cudaMemcpyHostToDevice, st));
    if (!symmetric) {
        if ((rc = upload(d_B, B, n))) return rc;
        NA_TRY_Q(cudaMemcpyAsync(d_bcB, bcB, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    }

    // The 128 x 256 tensor-core kernel where its accumulators are exact,
    // the popcount kernel otherwise; r^2 in the exact (FP64-evaluated) mode.
    const bool mma = (long long)K * 64 <= kMmaMaxSamples;
    const KernelShape &ks = mma ? kMmaShape : kPopcShape;
    CUtensorMap tmA, tmB;
    if (!make_map(&tmA, d_A, m, K, Kp, ks, true) || !make_map(&tmB, d_B, n, K, Kp, ks, false)) {
        cudaStreamSynchronize(st);
        cudaGetLastError();
        return QLD_ERR_CUDA;
    }

    for (int b0 = 0; b0 < n; b0 += band) {
        const int b1 = b0 + band < n ? b0 + band : n;
        LdParams p{};
        p.m = m; p.n = n; p.K = K; p.S = S;
        p.symmetric = symmetric;
        p.tb0 = b0 / ks.bn;
        p.nk = (K + ks.box_words - 1) / ks.box_words;
        p.bcA = d_bcA; p.bcB = d_bcB;
        p.r2 = d_band; p.ldr = m; p.counts = nullptr; p.ldc = m; p.out_row0 = b0;
        p.status = status;
        p.timeout_cycles = 4000000000LL;
        const int tiles_b = (b1 - b0 + ks.bn - 1) / ks.bn;
        NA_TRY_Q(mma ? launch_mma(tmA, tmB, p, tiles_b, R2_EXACT, st)
                   : launch_popc(tmA, tmB, p, tiles_b, R2_EXACT, st));
        // Stream order keeps the next band's kernel behind this copy.
        if (!symmetric) {
            NA_TRY_Q(cudaMemcpyAsync(r2_out + (size_t)b0 * m, d_band, (size_t)(b1 - b0) * m * 4,
                                   cudaMemcpyDeviceToHost, st));
        } else {
            for (int r0 = b0; r0 < b1; r0 += 512) {
                const int r1 = r0 + 512 < b1 ? r0 + 512 : b1;
                NA_TRY_Q(cudaMemcpy2DAsync(r2_out + (size_t)r0 * m + r0, (size_t)m * 4,
                                         d_band + (size_t)(r0 - b0) * m + r0, (size_t)m * 4,
                                         (size_t)(m - r0) * 4, r1 - r0, cudaMemcpyDeviceToHost,
                                         st));
            }
        }
    }
    unsigned h_status = 0;
    NA_TRY_Q(cudaMemcpyAsync(&h_status, status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    NA_TRY_Q(cudaStreamSynchronize(st));
    return h_status ? QLD_ERR_TIMEOUT : QLD_OK;
}
