// ld_mma.cu -- counts kernel, variant (b): bits unpacked to int8 {0,1} in
// shared memory, contracted by the 5th-generation tensor cores
// (tcgen05.mma.kind::i8, unsigned 8-bit operands, s32 accumulators in TMEM).
// Exact: every product is 0 or 1 and a count is at most the sample size
// (< 2^31).  The r^2 epilogue (qLD gemm_cpu.c:343-404) runs on the
// accumulators as they leave TMEM.  Same contraction as variant (a):
// qLD's blis_gemm()/bin_gemm_2x2 (gemm_cpu.c:125-341,
// blis/config/binary_gemm/kernels/3/bin_gemm.c:4-141).
//
// One CTA computes a 128 (A rows) x 256 (B rows) output tile.  Warp roles:
//   warp 0       TMA producer: per packed stage, 8 words (512 samples) of the
//                128 A rows and of the 256 B rows (64-byte swizzle), into a
//                ring of PST stages.
//   warp 1       TMEM allocation (256 columns) and the single MMA-issuing
//                thread: per unpacked stage (128 samples) 4 MMAs of
//                128 x 256 x 32, then tcgen05.commit to free the stage.
//   warps 2-9    unpack: each packed stage gives 4 unpacked stages of
//                128 A + 256 B rows x 128 bytes, written in the canonical
//                K-major 128-byte-swizzled layout the MMA descriptors name;
//                then the epilogue: tcgen05.ld of the accumulators, r^2,
//                coalesced stores (32 lanes = 32 consecutive A rows).
//
// Unpack mapping.  The 16 packed bytes of a row for one unpacked stage are
// four 32-bit words w0..w3; output 16-byte chunk c (c = 0..7) holds the
// words ((w0 >> c) & 0x01010101, ..., (w3 >> c) & 0x01010101), i.e. byte b of
// its word j is bit c + 8b of w_j.  This is a fixed permutation of the 128
// samples, the same for A and B, so sum_k a_k b_k is unchanged: one shift and
// one AND per 4 output bytes.
#include "qld_device.cuh"
#include "qld_kernels.h"

namespace qld {

namespace {

constexpr int BM = 128, BN = 256;
constexpr int PW = 8;                    // packed words per row per packed stage
constexpr int SUB = PW / 2;              // unpacked stages (128 samples) per packed stage
constexpr int PST = 4;                   // packed ring depth
constexpr int UST = 2;                   // unpacked ring depth
constexpr int PA_BYTES = BM * PW * 8;    // 8 KB
constexpr int PB_BYTES = BN * PW * 8;    // 16 KB
constexpr int UA_BYTES = BM * 128;       // 16 KB
constexpr int UB_BYTES = BN * 128;       // 32 KB
constexpr int UNPACK_WARPS = 8;
constexpr int UNPACK_THREADS = UNPACK_WARPS * 32;
constexpr int THREADS = 64 + UNPACK_THREADS;
constexpr uint32_t TMEM_COLS = 256;

// smem map (offsets from a 1024-byte aligned base)
constexpr int OFF_UA = 0;
constexpr int OFF_UB = OFF_UA + UST * UA_BYTES;
constexpr int OFF_PA = OFF_UB + UST * UB_BYTES;
constexpr int OFF_PB = OFF_PA + PST * PA_BYTES;
constexpr int OFF_BAR = OFF_PB + PST * PB_BYTES;
constexpr int NBARS = 2 * PST + 2 * UST + 1;
constexpr int OFF_TMEM = OFF_BAR + NBARS * 8;
constexpr int OFF_ROWS = (OFF_TMEM + 16 + 15) / 16 * 16;        // per-B-row epilogue factors
constexpr int ROWS_BYTES = BN * (8 + 4 + 4);
constexpr int SMEM_BYTES = OFF_ROWS + ROWS_BYTES + 1024;

// Instruction descriptor, kind::i8: D = s32 (bits 4-5 = 2), A and B unsigned
// 8-bit (bits 7-9, 10-12 = 0), both K-major (bits 15, 16 = 0),
// N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t IDESC = (2u << 4) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

// Shared-memory matrix descriptor for a K-major operand in the 128-byte
// swizzled canonical layout: rows of 128 bytes, 8-row atoms 1024 bytes apart
// (stride byte offset), fixed-constant bit 46, swizzle mode 2 (128 B).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;                       // leading byte offset (unused, 16 B)
    d |= (uint64_t)(1024u >> 4) << 32;             // stride byte offset
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_ld_32x32b_x32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
          "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
          "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ uint4 unpack_chunk(const uint4 &w, int c) {
    const uint32_t M = 0x01010101u;
    return make_uint4((w.x >> c) & M, (w.y >> c) & M, (w.z >> c) & M, (w.w >> c) & M);
}

template <int MODE>
__global__ void __launch_bounds__(THREADS, 1)
k_ld_mma(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
         const LdParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + OFF_BAR);
    uint64_t *pfull = bars, *pempty = bars + PST;
    uint64_t *ufull = bars + 2 * PST, *uempty = bars + 2 * PST + UST;
    uint64_t *accf = bars + 2 * PST + 2 * UST;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + OFF_TMEM);
    double *rowd = reinterpret_cast<double *>(smem + OFF_ROWS);
    uint32_t *rowc = reinterpret_cast<uint32_t *>(smem + OFF_ROWS + BN * 8);
    float *rowv = reinterpret_cast<float *>(smem + OFF_ROWS + BN * 12);

    const int ta = blockIdx.x;
    const int tb = p.tb0 + blockIdx.y;
    if (p.symmetric && ta * BM + BM - 1 < tb * BN) return;
    if (grid_failed(p.status)) return;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int np = (p.K + PW - 1) / PW;      // packed stages
    const int nu = np * SUB;                 // unpacked stages

    if (tid == 0) {
        for (int s = 0; s < PST; ++s) {
            mbar_init(smem_u32(&pfull[s]), 1);
            mbar_init(smem_u32(&pempty[s]), UNPACK_WARPS);
        }
        for (int s = 0; s < UST; ++s) {
            mbar_init(smem_u32(&ufull[s]), UNPACK_WARPS);
            mbar_init(smem_u32(&uempty[s]), 1);
        }
        mbar_init(smem_u32(accf), 1);
        fence_barrier_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // --------------------------------------------------------- producer --
        if (lane == 0) {
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            int issued = 0;
            for (int kp = 0; kp < np; ++kp) {
                const int s = kp % PST;
                if (kp >= PST && !mbar_wait(smem_u32(&pempty[s]), ((kp / PST) - 1) & 1,
                                            p.timeout_cycles, p.status)) {
                    flag_error(p.status, ST_TIMEOUT_EMPTY);
                    break;
                }
                const uint32_t fb = smem_u32(&pfull[s]);
                mbar_arrive_expect_tx(fb, PA_BYTES + PB_BYTES);
                tma_load_2d(smem_u32(smem + OFF_PA + s * PA_BYTES), &tmA, kp * PW, ta * BM, fb);
                tma_load_2d(smem_u32(smem + OFF_PB + s * PB_BYTES), &tmB, kp * PW, tb * BN, fb);
                ++issued;
            }
            for (int kp = issued > PST ? issued - PST : 0; kp < issued; ++kp)
                if (!mbar_wait(smem_u32(&pfull[kp % PST]), (kp / PST) & 1, p.timeout_cycles,
                               nullptr)) {
                    flag_error(p.status, ST_TIMEOUT_DRAIN);
                    break;
                }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------ MMA issuer --
        if (lane == 0) {
            for (int u = 0; u < nu; ++u) {
                const int s = u % UST;
                if (!mbar_wait(smem_u32(&ufull[s]), (u / UST) & 1, p.timeout_cycles, p.status)) {
                    flag_error(p.status, ST_TIMEOUT_UNPACK);
                    break;
                }
                tc_fence_after();
                const uint32_t a0 = smem_u32(smem + OFF_UA + s * UA_BYTES);
                const uint32_t b0 = smem_u32(smem + OFF_UB + s * UB_BYTES);
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                    tc_mma_i8(tmem, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32), IDESC,
                              (u > 0 || kk > 0) ? 1u : 0u);
                tc_commit(smem_u32(&uempty[s]));
            }
            // Fires once every MMA issued above has completed (also on the
            // error path, so TMEM is never released under a running MMA).
            tc_commit(smem_u32(accf));
        }
    } else {
        // --------------------------------------------------------- unpack --
        const int ut = tid - 64;
        // B-row epilogue factors for this tile, computed while data streams.
        {
            const int b = tb * BN + ut;
            const uint32_t c = b < p.n ? p.bcB[b] : 0u;
            rowc[ut] = c;
            if (MODE == R2_EXACT) {
                rowd[ut] = row_exact(c, p.S).inv_var;
            } else {
                const RowRef r = row_ref(c, p.S);
                rowv[ut] = r.v;
                rowd[ut] = r.one_minus;
            }
        }
        bool ok = true;
        for (int kp = 0; kp < np && ok; ++kp) {
            const int ps = kp % PST;
            // Wait outcomes are made warp-uniform so the warp never splits.
            const bool got = mbar_wait(smem_u32(&pfull[ps]), (kp / PST) & 1, p.timeout_cycles,
                                       p.status);
            if (!__all_sync(0xffffffffu, got)) {
                if (lane == 0) flag_error(p.status, ST_TIMEOUT_FULL);
                ok = false;
                break;
            }
            const uint8_t *pa = smem + OFF_PA + ps * PA_BYTES;
            const uint8_t *pb = smem + OFF_PB + ps * PB_BYTES;
            for (int sub = 0; sub < SUB; ++sub) {
                const int u = kp * SUB + sub;
                const int us = u % UST;
                const bool freed = u < UST || mbar_wait(smem_u32(&uempty[us]), ((u / UST) - 1) & 1,
                                                        p.timeout_cycles, p.status);
                if (!__all_sync(0xffffffffu, freed)) {
                    if (lane == 0) flag_error(p.status, ST_TIMEOUT_MMA);
                    ok = false;
                    break;
                }
                uint8_t *ua = smem + OFF_UA + us * UA_BYTES;
                uint8_t *ub = smem + OFF_UB + us * UB_BYTES;
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const int t = ut + j * UNPACK_THREADS;   // 768 tasks: (row, half)
                    const int row = t >> 1, half = t & 1;
                    const bool isA = row < BM;
                    const int r = isA ? row : row - BM;
                    // packed row r: 64 bytes, 64-byte swizzle (16-byte chunk ^= (r>>1)&3)
                    const uint8_t *src = (isA ? pa : pb) + r * 64 + ((sub ^ ((r >> 1) & 3)) << 4);
                    const uint4 w = *reinterpret_cast<const uint4 *>(src);
                    uint8_t *dst = (isA ? ua : ub) + r * 128;
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        const int c = half * 4 + cc;
                        *reinterpret_cast<uint4 *>(dst + ((c ^ (r & 7)) << 4)) = unpack_chunk(w, c);
                    }
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&ufull[us]));
            }
            if (!ok) break;
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&pempty[ps]));
        }

        // -------------------------------------------------------- epilogue --
        named_bar_sync(1, UNPACK_THREADS);   // row factors visible to all unpack warps
        bool ready = ok && mbar_wait(smem_u32(accf), 0, p.timeout_cycles, p.status);
        ready = __all_sync(0xffffffffu, ready);
        if (ready) {
            __syncwarp();
            tc_fence_after();
            const int q = warp & 3;                  // TMEM lane quarter of this warp
            const int h = (warp - 2) >> 2;           // column half
            const int a = ta * BM + q * 32 + lane;
            const bool a_ok = a < p.m;
            const uint32_t ca = a_ok ? p.bcA[a] : 0u;
            RowExact ra_e;
            RowRef ra_r;
            if (MODE == R2_EXACT) ra_e = row_exact(ca, p.S);
            else ra_r = row_ref(ca, p.S);
#pragma unroll 1
            for (int cb = 0; cb < 4; ++cb) {
                uint32_t v[32];
                const int col0 = h * 128 + cb * 32;
                __syncwarp();
                tc_ld_32x32b_x32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)col0, v);
#pragma unroll
                for (int t = 0; t < 32; ++t) {
                    const int bl = col0 + t;
                    const int b = tb * BN + bl;
                    if (b < p.n && a_ok && (!p.symmetric || a >= b)) {
                        float r2;
                        if (MODE == R2_EXACT) {
                            RowExact rb;
                            rb.c = rowc[bl];
                            rb.inv_var = rowd[bl];
                            r2 = r2_exact(v[t], ra_e, rb, p.S);
                        } else {
                            RowRef rb;
                            rb.c = rowc[bl];
                            rb.v = rowv[bl];
                            rb.one_minus = rowd[bl];
                            r2 = r2_reference(v[t], ra_r, rb, p.S);
                        }
                        const long long o = (long long)(b - p.out_row0);
                        p.r2[o * p.ldr + a] = r2;
                        if (p.counts) p.counts[o * p.ldc + a] = v[t];
                    }
                }
            }
        } else if (ok && lane == 0) {
            flag_error(p.status, ST_TIMEOUT_MMA);
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        // Every MMA must be complete before TMEM is released.
        if (!mbar_wait(smem_u32(accf), 0, p.timeout_cycles, nullptr))
            flag_error(p.status, ST_TIMEOUT_MMA);
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS)
                     : "memory");
    }
}

template <int MODE>
cudaError_t launch_mode(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                        int tiles_b, cudaStream_t st) {
    auto kern = k_ld_mma<MODE>;
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (e != cudaSuccess) return e;
    dim3 grid((p.m + BM - 1) / BM, tiles_b);
    kern<<<grid, THREADS, SMEM_BYTES, st>>>(tmA, tmB, p);
    return cudaGetLastError();
}

}  // namespace

// Both tensor maps use box_words = PW (64 bytes, 64-byte swizzle); A's box
// has BM rows, B's BN rows.
const KernelShape kMmaShape = {BM, BN, PW, BM, BN, 64};

cudaError_t launch_mma(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                       int tiles_b, int r2_mode, cudaStream_t st) {
    if (tiles_b <= 0 || p.m <= 0) return cudaSuccess;
    return r2_mode == R2_REFERENCE ? launch_mode<R2_REFERENCE>(tmA, tmB, p, tiles_b, st)
                                   : launch_mode<R2_EXACT>(tmA, tmB, p, tiles_b, st);
}

}  // namespace qld
