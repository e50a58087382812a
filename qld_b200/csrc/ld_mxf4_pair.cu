// ld_mxf4_pair.cu -- counts kernel, variant (c) on SM pairs: the 4-bit
// tensor-core path of ld_mxf4.cu (bits spread to E2M1 with normalising
// UE8M0 scale factors, tcgen05.mma.kind::mxf4 into F32 accumulators, exact
// below 2^24, FP32 r^2 epilogue)
// with every 256 x 240 output tile computed by a cluster of two CTAs on two
// SMs through tcgen05.mma.cta_group::2.
//
// Why pairs: one SM computing a 256 x 240 tile needs two 240-column
// accumulators, which with the scale factors fill its 512 TMEM columns, so
// the r^2 epilogue of a tile cannot overlap the MMAs of the next; and each
// of its two 128-row MMAs reads all 240 unpacked B rows.  Split over a pair,
// each SM holds 128 A rows and 120 B rows, one 128 x 240 accumulator per
// tile, and TMEM room for two of them: the epilogue warps drain one while
// the MMAs fill the other, and each SM's shared memory supplies every
// unpacked row once per MMA.
//
// Roles (both CTAs of a pair, 640 threads):
//   warp 0       TMA producer: the CTA's 128 A rows and 120 B rows, 8 packed
//                words (512 samples) per stage, 64-byte swizzle.
//   warp 1       TMEM allocation for the pair (cta_group::2); in rank 0 the
//                MMA issuer: per unpacked stage (256 samples) 4 MMAs of
//                256 x 240 x 64, then one commit that arrives on the stage's
//                "empty" barrier in both CTAs.
//   warps 2-11   unpack (w -> four words of nibbles, as ld_mxf4.cu) into the
//                CTA's stage; they arrive on rank 0's "full" barrier.  Two
//                groups of five warps take alternate unpacked stages (each
//                thread one or two rows of every other stage): two stages in
//                flight per CTA, which the per-warp latency of a stage (load,
//                spread, store, proxy fence, remote arrive) needs to keep up
//                with the MMAs.  Five warps per group measured 3 % faster than
//                four (2.44 / 2.76 ms against 2.52 / 2.83 ms, exact /
//                reference r^2); six, at the 80 registers 22 warps leave, 4 %
//                slower.
//   warps 12-19  epilogue: warp w reads TMEM lane quarter w % 4 of the
//                accumulator buffer the tile used, every other one of its
//                fifteen 16-column chunks, applies the r^2 epilogue (gemm_cpu.c:343-404) and
//                stores; they arrive on rank 0's "accumulator empty" barrier.
// Every wait is bounded.  No thread returns early: both CTAs meet at the
// cluster barriers at start and end on every path, including after a
// timeout, and the TMEM is released only after the last MMA has completed.
#include "epilogue.cuh"
#include "mxf4_rows.cuh"
#include "qld_kernels.h"
#include "tcgen05.cuh"

namespace qld {

namespace {

using namespace tc;

constexpr int BM = 256, BN = 240;        // output tile of a pair
constexpr int HM = 128, HN = 120;        // A and B rows held by each CTA
constexpr int PW = 8;                    // packed words per row per packed stage
constexpr int SUB = 2;                   // unpacked stages (256 samples) per packed stage
constexpr int UST = 4;
constexpr int PA_BYTES = HM * PW * 8;    // 8 KB
constexpr int PB_TX = HN * PW * 8;       // 7.5 KB delivered per stage
constexpr int PB_BYTES = 8192;           // stage stride, 1024-byte aligned
constexpr int UA_BYTES = HM * 128;       // 16 KB: 256 E2M1 per row
constexpr int UB_BYTES = HN * 128;       // 15 KB
constexpr int UNPACK_WARPS = 10, EPI_WARPS = 8;
constexpr int FIRST_UNPACK_WARP = 2;
constexpr int FIRST_EPI_WARP = FIRST_UNPACK_WARP + UNPACK_WARPS;
constexpr int EPILOGUE = EPI_WARPS * 32;
constexpr int THREADS = (FIRST_EPI_WARP + EPI_WARPS) * 32;   // 640
constexpr int GROUP_THREADS = UNPACK_WARPS * 32 / 2;         // unpackers per stage
constexpr int NTASK = HM + HN;                               // row tasks
constexpr int TASKS = (NTASK + GROUP_THREADS - 1) / GROUP_THREADS;
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t ACC_STRIDE = 256;     // accumulator buffers at columns 0 and 256
constexpr uint32_t SF_COL = 496;         // 16 columns of scale factors
constexpr uint32_t IDESC_EVEN = idesc_mxf4_sf(BM, BN, 0);   // k-steps 0, 2: scale bytes 0-1
constexpr uint32_t IDESC_ODD = idesc_mxf4_sf(BM, BN, 2);    // k-steps 1, 3: scale bytes 2-3
constexpr int COLS_N = 256;              // epilogue column factors (BN used)
constexpr uint16_t BOTH = 0x3;           // CTA mask of a commit to both ranks

// Shared-memory layout per r^2 mode.  R2_EXACT needs 8 bytes of column
// factors per column (epi::ColsF), R2_REFERENCE 16 (epi::ColsR); both leave
// room for six packed stages (more TMA lookahead than five: 2.576 -> 2.562
// ms on the single region).
template <int MODE>
struct Smem {
    static constexpr int PST = 6;                          // packed stages in flight
    static constexpr int OFF_UA = 0;
    static constexpr int OFF_UB = OFF_UA + UST * UA_BYTES;
    static constexpr int OFF_PA = OFF_UB + UST * UB_BYTES;
    static constexpr int OFF_PB = OFF_PA + PST * PA_BYTES;
    static constexpr int OFF_ROWS = OFF_PB + PST * PB_BYTES;
    static constexpr int ROWS_BYTES = COLS_N * (MODE == R2_EXACT ? 8 : epi::COLR_BYTES);
    static constexpr int OFF_BAR = OFF_ROWS + ROWS_BYTES;
    static constexpr int NBARS = 2 * PST + 2 * UST + 2 + 2 + 1;
    static constexpr int OFF_TMEM = OFF_BAR + NBARS * 8;
    static constexpr int BYTES = OFF_TMEM + 16 + 1024;
    static_assert(BYTES <= 232448, "shared memory budget");
    static_assert(OFF_UB % 1024 == 0 && UB_BYTES % 1024 == 0 && OFF_PA % 1024 == 0 &&
                      OFF_PB % 1024 == 0 && PB_TX <= PB_BYTES,
                  "swizzled stages must start on 1024-byte boundaries");
};
static_assert(sizeof(float2) == 8, "ColsF entry");
static_assert(ACC_STRIDE + BN <= SF_COL && SF_COL + 16 <= TMEM_COLS, "TMEM map");
static_assert(TASKS == 2 && SUB == 2 && UST % 2 == 0 && EPILOGUE == COLS_N, "work split");

template <int MODE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, 1)
k_ld_mxf4_pair(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
               const LdParams p, const int tiles_b) {
    using L = Smem<MODE>;
    constexpr int PST = L::PST;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::OFF_BAR);
    uint64_t *pfull = bars, *pempty = bars + PST;
    uint64_t *ufull = bars + 2 * PST, *uempty = bars + 2 * PST + UST;
    uint64_t *accfull = bars + 2 * PST + 2 * UST;
    uint64_t *accempty = accfull + 2;
    uint64_t *mma_done = accempty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L::OFF_TMEM);
    const epi::ColsR colsr(smem + L::OFF_ROWS, COLS_N);   // R2_REFERENCE factors
    const epi::ColsF colsf(smem + L::OFF_ROWS, COLS_N);   // R2_EXACT: FP32 factors

    const uint32_t rank = cluster_rank();
    const int pair = (int)cluster_id_x(), npairs = (int)cluster_count_x();
    const TileList<BM, BN> tl{(p.m + BM - 1) / BM, p.tb0, tiles_b, p.symmetric, p.band};
    const int dlo = diag_lo(p.symmetric, p.band), dhi = diag_hi(p.band);
    const int ntiles = tl.count();
    const int my_tiles = pair < ntiles ? (ntiles - pair + npairs - 1) / npairs : 0;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int np = (p.K + PW - 1) / PW;
    const int nu = np * SUB;

    if (tid == 0) {
        for (int s = 0; s < PST; ++s) {
            mbar_init(smem_u32(&pfull[s]), 1);
            mbar_init(smem_u32(&pempty[s]), UNPACK_WARPS);
        }
        for (int s = 0; s < UST; ++s) {
            mbar_init(smem_u32(&ufull[s]), UNPACK_WARPS);   // one group in each CTA
            mbar_init(smem_u32(&uempty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&accfull[b]), 1);
            mbar_init(smem_u32(&accempty[b]), 2 * EPI_WARPS);   // both CTAs' epilogues
        }
        mbar_init(smem_u32(mma_done), 1);
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc<2>(smem_u32(tmem_slot), TMEM_COLS);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // The spread's scale factors (kSpreadScales) in columns SF_COL.. of every
    // lane, in both CTAs; warps 2-5 cover the four TMEM lane quarters.
    if (warp >= FIRST_UNPACK_WARP && warp < FIRST_UNPACK_WARP + 4)
        tc_st_32x32b_x16_fill(tmem + ((uint32_t)((warp & 3) * 32) << 16) + SF_COL, kSpreadScales);
    tc_fence_before();
    // barrier initialisation and both CTAs' scale factors, cluster-wide
    cluster_sync_all();
    tc_fence_after();

    if (warp == 0) {
        // ------------------------------------------------------- producer --
        if (lane == 0) {
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            int gp = 0, cur_t = 0, cur_base = 0;
            bool ok = true;
            for (int i = 0; i < my_tiles && ok; ++i) {
                int ta, tb;
                tl.decode_from(pair + i * npairs, ta, tb, cur_t, cur_base);
                const int ra = ta * BM + (int)rank * HM, rb = tb * BN + (int)rank * HN;
                for (int kp = 0; kp < np; ++kp, ++gp) {
                    const int s = gp % PST;
                    if (gp >= PST && !mbar_wait(smem_u32(&pempty[s]), ((gp / PST) - 1) & 1,
                                                p.timeout_cycles, p.status)) {
                        flag_error(p.status, ST_TIMEOUT_EMPTY);
                        ok = false;
                        break;
                    }
                    const uint32_t fb = smem_u32(&pfull[s]);
                    mbar_arrive_expect_tx(fb, PA_BYTES + PB_TX);
                    tma_load_2d(smem_u32(smem + L::OFF_PA + s * PA_BYTES), &tmA, kp * PW, ra, fb);
                    tma_load_2d(smem_u32(smem + L::OFF_PB + s * PB_BYTES), &tmB, kp * PW, rb, fb);
                }
            }
            for (int g = gp > PST ? gp - PST : 0; g < gp; ++g)
                if (!mbar_wait(smem_u32(&pfull[g % PST]), (g / PST) & 1, kDrainCycles,
                               nullptr)) {
                    flag_error(p.status, ST_TIMEOUT_DRAIN);
                    break;
                }
        }
    } else if (warp == 1) {
        // ------------------------------------------- MMA issuer (rank 0) --
        if (lane == 0 && rank == 0) {
            const uint32_t sf = tmem + SF_COL;
            int gu = 0;
            bool ok = true;
            for (int it = 0; it < my_tiles && ok; ++it) {
                const int ab = it & 1;
                if (it >= 2 && !mbar_wait(smem_u32(&accempty[ab]), ((it >> 1) - 1) & 1,
                                                  p.timeout_cycles, p.status)) {
                    flag_error(p.status, ST_TIMEOUT_MMA);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)ab * ACC_STRIDE;
                for (int u = 0; u < nu; ++u, ++gu) {
                    const int s = gu % UST;
                    if (!mbar_wait(smem_u32(&ufull[s]), (gu / UST) & 1, p.timeout_cycles,
                                           p.status)) {
                        flag_error(p.status, ST_TIMEOUT_UNPACK);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(smem + L::OFF_UA + s * UA_BYTES);
                    const uint32_t b0 = smem_u32(smem + L::OFF_UB + s * UB_BYTES);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk)
                        tc_mma_mxf4_pair(d, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32),
                                         (kk & 1) ? IDESC_ODD : IDESC_EVEN,
                                         (u > 0 || kk > 0) ? 1u : 0u, sf, sf);
                    tc_commit_pair(smem_u32(&uempty[s]), BOTH);
                }
                tc_commit_pair(smem_u32(&accfull[ab]), BOTH);
            }
            tc_commit_pair(smem_u32(mma_done), BOTH);
        }
    } else if (warp < FIRST_EPI_WARP) {
        // --------------------------------------------------------- unpack --
        // group g takes the unpacked stages gu = g, g + 2, ...: sub-stage g of
        // every packed stage
        const int grp = (warp - FIRST_UNPACK_WARP) / (UNPACK_WARPS / 2);
        const int wt = ((warp - FIRST_UNPACK_WARP) % (UNPACK_WARPS / 2)) * 32 + lane;
        mxf4rows::RowTask task[TASKS];
#pragma unroll
        for (int j = 0; j < TASKS; ++j)   // over 128 A + 120 B rows
            task[j] = mxf4rows::make_task<HM>(wt + j * GROUP_THREADS, NTASK);
        const int total_u = my_tiles * nu;
        for (int gu = grp; gu < total_u; gu += 2) {
            const int gp = gu / SUB;
            const int ps = gp % PST;
            const bool got = mbar_wait(smem_u32(&pfull[ps]), (gp / PST) & 1, p.timeout_cycles,
                                       p.status);
            if (!__all_sync(0xffffffffu, got)) {
                if (lane == 0) flag_error(p.status, ST_TIMEOUT_FULL);
                break;
            }
            const int us = gu % UST;
            const bool freed = gu < UST || mbar_wait(smem_u32(&uempty[us]), ((gu / UST) - 1) & 1,
                                                     p.timeout_cycles, p.status);
            if (!__all_sync(0xffffffffu, freed)) {
                if (lane == 0) flag_error(p.status, ST_TIMEOUT_MMA);
                break;
            }
            mxf4rows::unpack_rows(task, smem + L::OFF_PA + ps * PA_BYTES, smem + L::OFF_PB + ps * PB_BYTES,
                        smem + L::OFF_UA + us * UA_BYTES, smem + L::OFF_UB + us * UB_BYTES, grp);
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_rank(smem_u32(&ufull[us]), 0);
                mbar_arrive(smem_u32(&pempty[ps]));     // both groups: UNPACK_WARPS per stage
            }
        }
    } else {
        // ------------------------------------------------------- epilogue --
        const int et = tid - FIRST_EPI_WARP * 32;
        const int ew = warp - FIRST_EPI_WARP;
        const int q = warp & 3;                 // TMEM lane quarter
        const int colh = ew >> 2;               // chunks colh, colh + 2, ... (< 15)
        bool failed = false;
        int cur_t = 0, cur_base = 0;
        for (int it = 0; it < my_tiles; ++it) {
            int ta, tb;
            tl.decode_from(pair + it * npairs, ta, tb, cur_t, cur_base);
            const int ab = it & 1;
            {   // every column factor the chunks read; 0 past the tile and the task
                const int b = tb * BN + et;
                const uint32_t cb = (et < BN && b < p.n) ? p.bcB[b] : 0u;
                if constexpr (MODE == R2_EXACT)
                    epi::store_col_f32(colsf, et, cb, p.S);
                else
                    epi::store_col_ref(colsr, et, cb, p.S);
            }
            named_bar_sync(1, EPILOGUE);
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
                const int a = ta * BM + (int)rank * HM + q * 32 + lane;
                const bool a_ok = a < p.m;
                const uint32_t ca = a_ok ? p.bcA[a] : 0u;
                const epi::ARowR ra = epi::make_arow_ref(ca, p.S);
                const epi::ARowF raf = epi::make_arow_f32(ca, p.S);
                const uint32_t tbase =
                    tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)ab * ACC_STRIDE;
                const int n_tile = tb * BN + BN < p.n ? tb * BN + BN : p.n;
                // 16-column chunks: fewer live registers than 32 (2.41 / 2.66 ms
                // against 2.43 / 2.75 ms, exact / reference r^2), the tile's 15
#pragma unroll 1
                for (int c = colh; c < BN / 16; c += 2) {
                    uint32_t v[16];
                    __syncwarp();
                    tc_ld_32x32b_x16(tbase + (uint32_t)(c * 16), v);
                    if constexpr (MODE == R2_EXACT) {
                        epi::chunk_f32<16>(v, tbase + (uint32_t)(c * 16), raf, colsf, c * 16,
                                           tb * BN + c * 16, a, a_ok, n_tile,
                                           dlo, dhi, p.r2, p.ldr, p.counts, p.ldc, p.out_row0, p.S);
                    } else {
                        // the F32 accumulators hold the counts as floats
                        epi::chunk_ref<0, true, 16>(v, ra, colsr, c * 16, tb * BN + c * 16, a, a_ok,
                                            n_tile, dlo, dhi, p.r2, p.ldr, p.counts, p.ldc,
                                            p.out_row0, p.S);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_rank(smem_u32(&accempty[ab]), 0);
            }
            named_bar_sync(1, EPILOGUE);
        }
    }

    // Teardown: the last commit of rank 0 arrives on mma_done in both CTAs;
    // neither CTA releases the pair's TMEM or exits while the other may
    // still touch its shared memory.
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        if (!mbar_wait(smem_u32(mma_done), 0, kDrainCycles, nullptr))
            flag_error(p.status, ST_TIMEOUT_MMA);
        __syncwarp();
    }
    tc_fence_before();
    cluster_sync_all();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc<2>(tmem, TMEM_COLS);
    }
}

int g_max_pairs = 0;

template <int MODE>
cudaError_t launch_mode(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                        int tiles_b, cudaStream_t st) {
    auto kern = k_ld_mxf4_pair<MODE>;
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Smem<MODE>::BYTES);
    if (e != cudaSuccess) return e;
    if (g_max_pairs == 0) {
        int dev = 0, sms = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) !=
            cudaSuccess)
            return e;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * (sms / 2), 1, 1);
        cfg.blockDim = dim3(THREADS, 1, 1);
        cfg.dynamicSmemBytes = Smem<MODE>::BYTES;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess || n <= 0) {
            (void)cudaGetLastError();
            n = sms / 2;
        }
        g_max_pairs = n;
    }
    const long long ntiles =
        TileList<BM, BN>{(p.m + BM - 1) / BM, p.tb0, tiles_b, p.symmetric, p.band}.count();
    if (ntiles == 0) return cudaSuccess;
    const int pairs = (int)(ntiles < g_max_pairs ? ntiles : g_max_pairs);
    kern<<<2 * pairs, THREADS, Smem<MODE>::BYTES, st>>>(tmA, tmB, p, tiles_b);
    return cudaGetLastError();
}

}  // namespace

const KernelShape kMxf4PairShape = {BM, BN, PW, HM, HN, 64};

cudaError_t launch_mxf4_pair(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                             int tiles_b, int r2_mode, cudaStream_t st) {
    if (tiles_b <= 0 || p.m <= 0) return cudaSuccess;
    return r2_mode == R2_REFERENCE ? launch_mode<R2_REFERENCE>(tmA, tmB, p, tiles_b, st)
                                   : launch_mode<R2_EXACT>(tmA, tmB, p, tiles_b, st);
}

}  // namespace qld
