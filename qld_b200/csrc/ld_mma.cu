// ld_mma.cu -- counts kernel, variant (b): bits unpacked to 8-bit {0, 0x80}
// in shared memory and contracted by the 5th-generation tensor cores
// (tcgen05.mma.kind::i8, unsigned 8-bit operands, s32 accumulators in TMEM).
// Every product is 0 or 0x80 * 0x80 = 2^14, so an accumulator holds exactly
// 2^14 * count, which fits in s32 while the sample count is below 2^17
// (the host routes larger K to variant (a)).  The r^2 epilogue (qLD
// gemm_cpu.c:343-404) runs on the accumulators as they leave TMEM.  Same
// contraction as variant (a): qLD's blis_gemm()/bin_gemm_2x2
// (gemm_cpu.c:125-341, blis/config/binary_gemm/kernels/3/bin_gemm.c:4-141).
//
// Persistent: one CTA per SM walks a static list of 128 (A rows) x 256
// (B rows) output tiles; tiles of a launch are ordered B-tile-row first so
// the CTAs running at the same time share B panels in L2.  Warp roles:
//   warp 0       TMA producer: per packed stage 8 words (512 samples) of the
//                tile's 128 A rows and 256 B rows (64-byte swizzle).
//   warp 1       TMEM owner (512 columns = two 128 x 256 s32 accumulators)
//                and the MMA-issuing thread: per unpacked stage (128
//                samples) 4 MMAs of 128 x 256 x 32 into the tile's
//                accumulator, tcgen05.commit frees the stage; after the
//                tile, a commit hands the accumulator to the epilogue.
//   warps 2-13   unpack: each packed stage gives 4 unpacked stages of
//                128 + 256 rows x 128 bytes in the canonical K-major
//                128-byte-swizzled layout the MMA descriptors name.
//   warps 14-17  epilogue: tcgen05.ld of the finished accumulator (warp w
//                reads TMEM lanes 32*(w%4)..), r^2, coalesced stores
//                (32 lanes = 32 consecutive A rows), then release the
//                accumulator -- overlapping the next tile's MMAs.
//
// Unpack mapping.  The 16 packed bytes of a row for one unpacked stage are
// four 32-bit words w0..w3; output 16-byte chunk c (c = 0..7) holds the
// words ((w0 << (7-c)) & 0x80808080, ..., (w3 << (7-c)) & 0x80808080), i.e.
// byte b of its word j carries bit c + 8b of w_j.  This is a fixed
// permutation of the 128 samples, the same for A and B, so the contraction
// is unchanged: one shift and one AND per 4 bytes.  The shift is written as
// a multiply by a per-thread power of two held in a register, so it runs on
// the IMAD pipe and leaves the ALU pipe to the ANDs.
#include "epilogue.cuh"
#include "qld_kernels.h"
#include "tcgen05.cuh"

namespace qld {

namespace {

using namespace tc;

constexpr int BM = 128, BN = 256;
constexpr int PW = 8;                    // packed words per row per packed stage
constexpr int SUB = PW / 2;              // unpacked stages (128 samples) per packed stage
constexpr int PST = 3;                   // packed ring depth
constexpr int UST = 3;                   // unpacked ring depth
constexpr int PA_BYTES = BM * PW * 8;    // 8 KB
constexpr int PB_BYTES = BN * PW * 8;    // 16 KB
constexpr int UA_BYTES = BM * 128;       // 16 KB
constexpr int UB_BYTES = BN * 128;       // 32 KB
constexpr int UNPACK_WARPS = 12;
constexpr int UNPACK_THREADS = UNPACK_WARPS * 32;
constexpr int EPI_WARPS = 4;
constexpr int EPI_THREADS = EPI_WARPS * 32;
constexpr int FIRST_UNPACK_WARP = 2;
constexpr int FIRST_EPI_WARP = FIRST_UNPACK_WARP + UNPACK_WARPS;
constexpr int THREADS = (FIRST_EPI_WARP + EPI_WARPS) * 32;   // 576
constexpr int TASKS = 2 * (BM + BN) / UNPACK_THREADS;           // (row, half) tasks per thread
static_assert(TASKS * UNPACK_THREADS == 2 * (BM + BN), "unpack tasks must divide evenly");
constexpr uint32_t TMEM_COLS = 512;                          // two accumulators

// smem map (offsets from a 1024-byte aligned base)
constexpr int OFF_UA = 0;
constexpr int OFF_UB = OFF_UA + UST * UA_BYTES;
constexpr int OFF_PA = OFF_UB + UST * UB_BYTES;
constexpr int OFF_PB = OFF_PA + PST * PA_BYTES;
constexpr int OFF_ROWS = OFF_PB + PST * PB_BYTES;            // per-B-row epilogue factors
constexpr int ROWS_BYTES = BN * epi::COL_BYTES;
constexpr int OFF_BAR = OFF_ROWS + ROWS_BYTES;
constexpr int NBARS = 2 * PST + 2 * UST + 2 + 2 + 1;
constexpr int OFF_TMEM = OFF_BAR + NBARS * 8;
constexpr int SMEM_BYTES = OFF_TMEM + 16 + 1024;
static_assert(SMEM_BYTES <= 232448, "shared memory budget");

constexpr uint32_t IDESC = tc::idesc_i8(BM, BN);

template <int MODE>
__global__ void __launch_bounds__(THREADS, 1)
k_ld_mma(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
         const LdParams p, const int tiles_b) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + OFF_BAR);
    uint64_t *pfull = bars, *pempty = bars + PST;
    uint64_t *ufull = bars + 2 * PST, *uempty = bars + 2 * PST + UST;
    uint64_t *accfull = bars + 2 * PST + 2 * UST;
    uint64_t *accempty = accfull + 2;
    uint64_t *mma_done = accempty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + OFF_TMEM);
    const epi::Cols cols(smem + OFF_ROWS, BN);

    if (grid_failed(p.status)) return;
    const TileList<BM, BN> tl{(p.m + BM - 1) / BM, p.tb0, tiles_b, p.symmetric, p.band};
    const int dlo = diag_lo(p.symmetric, p.band), dhi = diag_hi(p.band);
    const int ntiles = tl.count();
    if ((int)blockIdx.x >= ntiles) return;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int np = (p.K + PW - 1) / PW;      // packed stages per tile

    if (tid == 0) {
        for (int s = 0; s < PST; ++s) {
            mbar_init(smem_u32(&pfull[s]), 1);
            mbar_init(smem_u32(&pempty[s]), UNPACK_WARPS);
        }
        for (int s = 0; s < UST; ++s) {
            mbar_init(smem_u32(&ufull[s]), UNPACK_WARPS);
            mbar_init(smem_u32(&uempty[s]), 1);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(smem_u32(&accfull[s]), 1);
            mbar_init(smem_u32(&accempty[s]), EPI_WARPS);
        }
        mbar_init(smem_u32(mma_done), 1);
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc<1>(smem_u32(tmem_slot), TMEM_COLS);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------- producer --
        if (lane == 0) {
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            int gp = 0;   // packed stages issued so far (ring position)
            bool ok = true;
            int cur_t = 0, cur_base = 0;   // decode_from: tiles in increasing order
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                int ta, tb;
                tl.decode_from(tile, ta, tb, cur_t, cur_base);
                for (int kp = 0; kp < np; ++kp, ++gp) {
                    const int s = gp % PST;
                    if (gp >= PST && !mbar_wait(smem_u32(&pempty[s]), ((gp / PST) - 1) & 1,
                                                p.timeout_cycles, p.status)) {
                        flag_error(p.status, ST_TIMEOUT_EMPTY);
                        ok = false;
                        break;
                    }
                    const uint32_t fb = smem_u32(&pfull[s]);
                    mbar_arrive_expect_tx(fb, PA_BYTES + PB_BYTES);
                    tma_load_2d(smem_u32(smem + OFF_PA + s * PA_BYTES), &tmA, kp * PW, ta * BM, fb);
                    tma_load_2d(smem_u32(smem + OFF_PB + s * PB_BYTES), &tmB, kp * PW, tb * BN, fb);
                }
            }
            // Drain: this CTA's copies must land before it retires.
            for (int g = gp > PST ? gp - PST : 0; g < gp; ++g)
                if (!mbar_wait(smem_u32(&pfull[g % PST]), (g / PST) & 1, kDrainCycles,
                               nullptr)) {
                    flag_error(p.status, ST_TIMEOUT_DRAIN);
                    break;
                }
        }
    } else if (warp == 1) {
        // ----------------------------------------------------- MMA issuer --
        if (lane == 0) {
            int gu = 0, it = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++it) {
                const int ab = it & 1;
                if (it >= 2 && !mbar_wait(smem_u32(&accempty[ab]), ((it >> 1) - 1) & 1,
                                          p.timeout_cycles, p.status)) {
                    flag_error(p.status, ST_TIMEOUT_MMA);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(ab * BN);
                for (int u = 0; u < np * SUB; ++u, ++gu) {
                    const int s = gu % UST;
                    if (!mbar_wait(smem_u32(&ufull[s]), (gu / UST) & 1, p.timeout_cycles,
                                   p.status)) {
                        flag_error(p.status, ST_TIMEOUT_UNPACK);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(smem + OFF_UA + s * UA_BYTES);
                    const uint32_t b0 = smem_u32(smem + OFF_UB + s * UB_BYTES);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                        tc_mma_i8(d, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32), IDESC,
                                  (u > 0 || kk > 0) ? 1u : 0u);
                    tc_commit(smem_u32(&uempty[s]));
                }
                tc_commit(smem_u32(&accfull[ab]));   // also on the error path
            }
            tc_commit(smem_u32(mma_done));           // every MMA above has completed
        }
    } else if (warp < FIRST_EPI_WARP) {
        // --------------------------------------------------------- unpack --
        const int ut = tid - FIRST_UNPACK_WARP * 32;
        UnpackTask task[TASKS];
#pragma unroll
        for (int j = 0; j < TASKS; ++j) {
            const int t = ut + j * UNPACK_THREADS;   // (row, half) over 128 A + 256 B rows
            const int row = t >> 1, half = t & 1;
            const bool isA = row < BM;
            const int r = isA ? row : row - BM;
            task[j].is_a = isA;
            task[j].src = (uint32_t)(r * 64);
            task[j].xr = (uint32_t)((r >> 1) & 3);
            task[j].dst = (uint32_t)(r * 128);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                const int c = half * 4 + cc;
                task[j].chunk_off[cc] = (uint32_t)((c ^ (r & 7)) << 4);
                task[j].pow2[cc] = 1u << (7 - c);
            }
        }
        int gp = 0, gu = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
            for (int kp = 0; kp < np && ok; ++kp, ++gp) {
                const int ps = gp % PST;
                // Wait outcomes are made warp-uniform so the warp never splits.
                const bool got = mbar_wait(smem_u32(&pfull[ps]), (gp / PST) & 1,
                                           p.timeout_cycles, p.status);
                if (!__all_sync(0xffffffffu, got)) {
                    if (lane == 0) flag_error(p.status, ST_TIMEOUT_FULL);
                    ok = false;
                    break;
                }
                const uint8_t *pa = smem + OFF_PA + ps * PA_BYTES;
                const uint8_t *pb = smem + OFF_PB + ps * PB_BYTES;
                for (int sub = 0; sub < SUB; ++sub, ++gu) {
                    const int us = gu % UST;
                    const bool freed = gu < UST || mbar_wait(smem_u32(&uempty[us]),
                                                             ((gu / UST) - 1) & 1,
                                                             p.timeout_cycles, p.status);
                    if (!__all_sync(0xffffffffu, freed)) {
                        if (lane == 0) flag_error(p.status, ST_TIMEOUT_MMA);
                        ok = false;
                        break;
                    }
                    uint8_t *ua = smem + OFF_UA + us * UA_BYTES;
                    uint8_t *ub = smem + OFF_UB + us * UB_BYTES;
                    uint4 w[TASKS];
#pragma unroll
                    for (int j = 0; j < TASKS; ++j)
                        w[j] = *reinterpret_cast<const uint4 *>(
                            (task[j].is_a ? pa : pb) + task[j].src + ((sub ^ task[j].xr) << 4));
#pragma unroll
                    for (int j = 0; j < TASKS; ++j) {
                        uint8_t *dst = (task[j].is_a ? ua : ub) + task[j].dst;
#pragma unroll
                        for (int cc = 0; cc < 4; ++cc)
                            *reinterpret_cast<uint4 *>(dst + task[j].chunk_off[cc]) =
                                unpack_chunk(w[j], task[j].pow2[cc]);
                    }
                    fence_proxy_async_smem();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(smem_u32(&ufull[us]));
                }
                if (!ok) break;
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&pempty[ps]));
            }
        }
    } else {
        // ------------------------------------------------------- epilogue --
        const int et = tid - FIRST_EPI_WARP * 32;
        const int q = warp & 3;                  // TMEM lane quarter of this warp
        bool failed = false;
        int it = 0;
        int cur_t = 0, cur_base = 0;   // decode_from: tiles in increasing order
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            int ta, tb;
            tl.decode_from(tile, ta, tb, cur_t, cur_base);
            const int ab = it & 1;
            // B-row factors of this tile: 2 per thread.
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int bl = et + k * EPI_THREADS;
                const int b = tb * BN + bl;
                epi::store_col<MODE>(cols, bl, b < p.n ? p.bcB[b] : 0u, p.S);
            }
            named_bar_sync(1, EPI_THREADS);
            // On a failed wait the warp skips the tile but stays in the loop,
            // so all four epilogue warps keep meeting at the named barrier
            // (later waits fail fast once the status word is set).
            bool ready = !failed && mbar_wait(smem_u32(&accfull[ab]), (it >> 1) & 1,
                                              p.timeout_cycles, p.status);
            ready = __all_sync(0xffffffffu, ready);
            if (!ready && !failed) {
                if (lane == 0) flag_error(p.status, ST_TIMEOUT_MMA);
                failed = true;
            }
            if (ready) {
                __syncwarp();
                tc_fence_after();
                const int a = ta * BM + q * 32 + lane;
                const bool a_ok = a < p.m;
                const epi::ARow ra = epi::make_arow<MODE>(a_ok ? p.bcA[a] : 0u, p.S);
                const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * BN);
#pragma unroll 1
                for (int col0 = 0; col0 < BN; col0 += 32) {
                    uint32_t v[32];
                    __syncwarp();
                    tc_ld_32x32b_x32(tbase + (uint32_t)col0, v);
                    epi::chunk<MODE, COUNT_SHIFT>(v, ra, cols, col0, tb * BN + col0, a, a_ok,
                                                  p.n, dlo, dhi, p.r2, p.ldr, p.counts, p.ldc,
                                                  p.out_row0, p.S);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&accempty[ab]));
            }
            named_bar_sync(1, EPI_THREADS);   // row factors may be rewritten
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        // Every MMA must be complete before TMEM is released.
        if (!mbar_wait(smem_u32(mma_done), 0, kDrainCycles, nullptr))
            flag_error(p.status, ST_TIMEOUT_MMA);
        __syncwarp();
        tc_fence_after();
        tmem_dealloc<1>(tmem, TMEM_COLS);
    }
}

int g_sm_count = 0;

template <int MODE>
cudaError_t launch_mode(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                        int tiles_b, cudaStream_t st) {
    auto kern = k_ld_mma<MODE>;
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (e != cudaSuccess) return e;
    if (g_sm_count == 0) {
        int dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev)) !=
            cudaSuccess)
            return e;
    }
    const long long ntiles =
        TileList<BM, BN>{(p.m + BM - 1) / BM, p.tb0, tiles_b, p.symmetric, p.band}.count();
    if (ntiles == 0) return cudaSuccess;
    const int grid = (int)(ntiles < g_sm_count ? ntiles : g_sm_count);
    kern<<<grid, THREADS, SMEM_BYTES, st>>>(tmA, tmB, p, tiles_b);
    return cudaGetLastError();
}

}  // namespace

// Both tensor maps use box_words = PW (64 bytes, 64-byte swizzle); A's box
// has BM rows, B's BN rows.
const KernelShape kMmaShape = {BM, BN, PW, BM, BN, 64};
const int kMmaMaxSamples = (1 << (31 - COUNT_SHIFT)) - 1;

cudaError_t launch_mma(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                       int tiles_b, int r2_mode, cudaStream_t st) {
    if (tiles_b <= 0 || p.m <= 0) return cudaSuccess;
    return r2_mode == R2_REFERENCE ? launch_mode<R2_REFERENCE>(tmA, tmB, p, tiles_b, st)
                                   : launch_mode<R2_EXACT>(tmA, tmB, p, tiles_b, st);
}

}  // namespace qld
