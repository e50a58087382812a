// ld_batch.cu -- many independent LD tasks (region pairs of uneven SNP and
// sample counts) in one persistent launch fed by a device work queue.
//
// Per-task arithmetic is that of the 4-bit kernels on SM pairs
// (ld_mxf4_pair.cu): bits spread to E2M1 with normalising UE8M0 scale
// factors (tcgen05.cuh: spread_e2m1), tcgen05.mma.cta_group::2.kind::mxf4
// into F32 TMEM accumulators that hold the counts exactly (K * 64 <= 2^24),
// fused r^2 epilogue of qLD gemm_cpu.c:343-404 (R2_EXACT in FP32 from the
// exact counts, epilogue.cuh: chunk_f32).  qLD itself runs such task lists
// one task at a time (-inputList, src/correlator/src/input_list.c:205-323
// and correlate_function.c:59-83).  Here every 256 x 240 output tile of every
// task is a work item, computed by a cluster of two CTAs (rank r: A rows
// 128 r.., B rows 120 r.. of the tile).  The device job table holds per task
// its tensor maps, sizes and output, and the item prefix offsets; items are
// numbered task by task (tasks sorted by cost on the host, most expensive
// first).
//
// Work queue: rank 0's producer thread claims the next item with an atomic
// ticket on a global counter, decodes it into (task, A tile, B tile) and
// writes it into the 4-slot item ring of both CTAs (the peer's copy through
// st.shared::cluster, published by a cluster-scope release arrive).  In each
// CTA the TMA thread, the unpack warps and the epilogue warps (and in rank 0
// the MMA thread) pop the same items in the same order, and each releases
// the slot on rank 0's barrier when done with its item.  A ticket past the
// last item pushes an end marker.
//
// Roles per CTA (576 threads in R2_EXACT, 704 in R2_REFERENCE): warp 0 queue
// (rank 0) and TMA of the CTA's rows, warp 1 TMEM and (rank 0) the MMAs,
// warps 2-9 unpack in two groups taking alternate 256-sample stages (each
// thread whole rows), warps 10-17 (10-21) epilogue, two (three) per TMEM lane
// quarter.  TMEM: two 240-column accumulators
// (columns 0 and 256), so a tile's epilogue overlaps the next tile's MMAs,
// and the scale factors at columns 496-511.  Every wait is bounded and no
// thread returns early: both CTAs meet at the cluster barriers at start and
// end on every path.
#include "epilogue.cuh"
#include "mxf4_rows.cuh"
#include "qld_kernels.h"
#include "tcgen05.cuh"

namespace qld {

namespace {

using namespace tc;

constexpr int BM = 256, BN = 240;           // work item: output tile of a pair
constexpr int HM = 128, HN = 120;           // A and B rows held by each CTA
constexpr int PW = 8;                       // packed words per row per packed stage
constexpr int SUB = 2;                      // unpacked stages (256 samples) per packed stage
constexpr int UST = 4;                      // two unpacked stages per unpack group
constexpr int PA_BYTES = HM * PW * 8;       // 8 KB
constexpr int PB_TX = HN * PW * 8;          // 7.5 KB delivered per stage
constexpr int PB_BYTES = 8192;              // stage stride, 1024-byte aligned
constexpr int UA_BYTES = HM * 128;          // 16 KB: 256 E2M1 per row
constexpr int UB_BYTES = HN * 128;          // 15 KB
constexpr int UNPACK_WARPS = 8;
constexpr int GROUP_THREADS = UNPACK_WARPS * 32 / 2;
constexpr int FIRST_UNPACK_WARP = 2;
constexpr int FIRST_EPI_WARP = FIRST_UNPACK_WARP + UNPACK_WARPS;
constexpr int NROWS = HM + HN;                                // row tasks per stage
constexpr int TASKS = (NROWS + GROUP_THREADS - 1) / GROUP_THREADS;
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t ACC_STRIDE = 256;
constexpr uint32_t SF_COL = 496;
constexpr uint32_t IDESC_EVEN = idesc_mxf4_sf(BM, BN, 0);   // k-steps 0, 2: scale bytes 0-1
constexpr uint32_t IDESC_ODD = idesc_mxf4_sf(BM, BN, 2);    // k-steps 1, 3: scale bytes 2-3
constexpr int COLS_N = 256;                                  // epilogue column factors (BN used)
constexpr uint16_t BOTH = 0x3;                               // CTA mask of a commit to both ranks
constexpr int QSLOTS = 4;                                    // item ring depth
// arrivals on rank 0's slot-free barrier per item: rank 0's MMA thread,
// unpack and epilogue warps; rank 1's TMA thread, unpack and epilogue warps
// Epilogue warps per r^2 mode: eight in R2_EXACT, twelve in R2_REFERENCE,
// whose longer per-pair sequence leaves items below ~6,000 samples waiting
// on their epilogue (4,096-task mix, reference mode: 87.7 against 95.0 ms;
// exact mode with twelve: 72.1 against 69.2 ms, its 32-column chunks spill
// at the 80 registers 704 threads leave).
template <int MODE>
struct Roles {
    static constexpr int EPI_WARPS = MODE == R2_REFERENCE ? 12 : 8;
    static constexpr int EPI_THREADS = EPI_WARPS * 32;
    static constexpr int THREADS = (FIRST_EPI_WARP + EPI_WARPS) * 32;   // 576 or 704
    static constexpr int ITEM_USERS = 2 * (1 + UNPACK_WARPS + EPI_WARPS);
    static_assert(EPI_WARPS % 4 == 0 && EPI_THREADS >= COLS_N, "epilogue split");
};

// Shared-memory layout per r^2 mode: R2_EXACT needs 8 bytes of column
// factors per column (epi::ColsF), R2_REFERENCE 16 (epi::ColsR); both leave
// room for six packed stages (more TMA lookahead than five).
template <int MODE>
struct Smem {
    static constexpr int PST = 6;                          // packed stages in flight
    static constexpr int OFF_UA = 0;
    static constexpr int OFF_UB = OFF_UA + UST * UA_BYTES;
    static constexpr int OFF_PA = OFF_UB + UST * UB_BYTES;
    static constexpr int OFF_PB = OFF_PA + PST * PA_BYTES;
    static constexpr int OFF_ROWS = OFF_PB + PST * PB_BYTES;
    static constexpr int ROWS_BYTES = COLS_N * (MODE == R2_EXACT ? 8 : epi::COLR_BYTES);
    static constexpr int OFF_ITEMS = OFF_ROWS + ROWS_BYTES;
    static constexpr int OFF_BAR = OFF_ITEMS + QSLOTS * 16;
    static constexpr int NBARS = 2 * PST + 2 * UST + 2 + 2 + 1 + 2 * QSLOTS;
    static constexpr int OFF_TMEM = OFF_BAR + NBARS * 8;
    static constexpr int BYTES = OFF_TMEM + 16 + 1024;
    static_assert(BYTES <= 232448, "shared memory budget");
    static_assert(OFF_UB % 1024 == 0 && UB_BYTES % 1024 == 0 && OFF_PA % 1024 == 0 &&
                      OFF_PB % 1024 == 0 && PB_TX <= PB_BYTES && OFF_ITEMS % 16 == 0,
                  "swizzled stages must start on 1024-byte boundaries");
};
static_assert(ACC_STRIDE + BN <= SF_COL && SF_COL + 16 <= TMEM_COLS, "TMEM map");
static_assert(TASKS == 2 && SUB == 2 && UST % 2 == 0, "work split");

struct Item {
    int job, ta, tb, np;   // job < 0: end of the queue
};
static_assert(sizeof(Item) == 16, "an item is one 16-byte record");

// (job, ta, tb) of global item g: binary search of the item prefix, then the
// job's own B-tile-row-first tile list.
__device__ __forceinline__ Item decode_item(const BatchJob *jobs, int njobs, long long g) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].item0 <= g) lo = mid;
        else hi = mid - 1;
    }
    const BatchJob &J = jobs[lo];
    const TileList<BM, BN> tl{(J.m + BM - 1) / BM, 0, (J.n + BN - 1) / BN, J.symmetric, 0};
    Item it;
    it.job = lo;
    tl.decode((int)(g - J.item0), it.ta, it.tb);
    it.np = (J.K + PW - 1) / PW;
    return it;
}

template <int MODE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(Roles<MODE>::THREADS, 1)
k_ld_batch(const BatchParams bp) {
    using L = Smem<MODE>;
    using R = Roles<MODE>;
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
    uint64_t *ifull = mma_done + 1, *iempty = ifull + QSLOTS;
    Item *items = reinterpret_cast<Item *>(smem + L::OFF_ITEMS);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L::OFF_TMEM);
    const epi::ColsR colsr(smem + L::OFF_ROWS, COLS_N);   // R2_REFERENCE factors
    const epi::ColsF colsf(smem + L::OFF_ROWS, COLS_N);   // R2_EXACT: FP32 factors

    const uint32_t rank = cluster_rank();
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const long long limit = bp.timeout_cycles;
    // the item ring is written by rank 0; rank 1 reads it under cluster-scope acquire
    auto wait_item = [&](int qi) {
        const uint32_t b = smem_u32(&ifull[qi % QSLOTS]);
        const uint32_t par = (uint32_t)(qi / QSLOTS) & 1u;
        return rank == 0 ? mbar_wait(b, par, limit, bp.status)
                         : mbar_wait_acq_cluster(b, par, limit, bp.status);
    };
    auto release_item = [&](int qi) { mbar_arrive_rank(smem_u32(&iempty[qi % QSLOTS]), 0); };

    if (tid == 0) {
        for (int s = 0; s < PST; ++s) {
            mbar_init(smem_u32(&pfull[s]), 1);
            mbar_init(smem_u32(&pempty[s]), UNPACK_WARPS);   // both groups, once each
        }
        for (int s = 0; s < UST; ++s) {
            mbar_init(smem_u32(&ufull[s]), UNPACK_WARPS);    // one group in each CTA
            mbar_init(smem_u32(&uempty[s]), 1);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(smem_u32(&accfull[s]), 1);
            mbar_init(smem_u32(&accempty[s]), 2 * R::EPI_WARPS);   // both CTAs' epilogues
        }
        mbar_init(smem_u32(mma_done), 1);
        for (int s = 0; s < QSLOTS; ++s) {
            mbar_init(smem_u32(&ifull[s]), 1);
            mbar_init(smem_u32(&iempty[s]), R::ITEM_USERS);
        }
        fence_barrier_init();
    }
    if (warp == 1) {
        tmem_alloc<2>(smem_u32(tmem_slot), TMEM_COLS);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // the spread's scale factors in columns SF_COL.. of every lane, in both
    // CTAs (warps 2-5 cover the four TMEM lane quarters)
    if (warp >= FIRST_UNPACK_WARP && warp < FIRST_UNPACK_WARP + 4)
        tc_st_32x32b_x16_fill(tmem + ((uint32_t)((warp & 3) * 32) << 16) + SF_COL, kSpreadScales);
    tc_fence_before();
    // barrier initialisation and both CTAs' scale factors, cluster-wide
    cluster_sync_all();
    tc_fence_after();

    if (warp == 0) {
        // ------------------------------- work queue (rank 0) + TMA producer --
        if (lane == 0) {
            int gp = 0;
            bool ok = true;
            for (int qi = 0;; ++qi) {
                const int slot = qi % QSLOTS;
                Item it;
                if (rank == 0) {
                    if (qi >= QSLOTS &&
                        !mbar_wait_acq_cluster(smem_u32(&iempty[slot]), ((qi / QSLOTS) - 1) & 1,
                                               limit, bp.status)) {
                        flag_error(bp.status, ST_TIMEOUT_EMPTY);
                        ok = false;
                    }
                    const long long g =
                        ok ? (long long)atomicAdd(bp.queue, 1ull) : (long long)bp.nitems;
                    if (g < bp.nitems) it = decode_item(bp.jobs, bp.njobs, g);
                    else it.job = -1, it.ta = it.tb = it.np = 0;
                    items[slot] = it;
                    mbar_arrive(smem_u32(&ifull[slot]));   // release: the item is visible
                    st_rank_and_arrive(smem_u32(&items[slot]),
                                       make_int4(it.job, it.ta, it.tb, it.np),
                                       smem_u32(&ifull[slot]), 1);
                } else {
                    if (!wait_item(qi)) {
                        flag_error(bp.status, ST_TIMEOUT_FULL);
                        break;
                    }
                    it = items[slot];
                }
                if (it.job < 0) break;
                const BatchJob &J = bp.jobs[it.job];
                const int ra = it.ta * BM + (int)rank * HM, rb = it.tb * BN + (int)rank * HN;
                for (int kp = 0; kp < it.np && ok; ++kp, ++gp) {
                    const int s = gp % PST;
                    if (gp >= PST && !mbar_wait(smem_u32(&pempty[s]), ((gp / PST) - 1) & 1,
                                                limit, bp.status)) {
                        flag_error(bp.status, ST_TIMEOUT_EMPTY);
                        ok = false;
                        break;
                    }
                    const uint32_t fb = smem_u32(&pfull[s]);
                    mbar_arrive_expect_tx(fb, PA_BYTES + PB_TX);
                    tma_load_2d(smem_u32(smem + L::OFF_PA + s * PA_BYTES), &J.tmA, kp * PW, ra, fb);
                    tma_load_2d(smem_u32(smem + L::OFF_PB + s * PB_BYTES), &J.tmB, kp * PW, rb, fb);
                }
                if (rank == 1) {
                    release_item(qi);
                    if (!ok) break;
                }
            }
            for (int g = gp > PST ? gp - PST : 0; g < gp; ++g)
                if (!mbar_wait(smem_u32(&pfull[g % PST]), (g / PST) & 1, kDrainCycles, nullptr)) {
                    flag_error(bp.status, ST_TIMEOUT_DRAIN);
                    break;
                }
        }
    } else if (warp == 1) {
        // ------------------------------------------- MMA issuer (rank 0) --
        if (lane == 0 && rank == 0) {
            const uint32_t sf = tmem + SF_COL;
            int gu = 0, it_n = 0;
            bool ok = true;
            for (int qi = 0; ok; ++qi, ++it_n) {
                const int slot = qi % QSLOTS;
                if (!wait_item(qi)) {
                    flag_error(bp.status, ST_TIMEOUT_UNPACK);
                    break;
                }
                const Item it = items[slot];
                if (it.job < 0) break;
                const int ab = it_n & 1;
                if (it_n >= 2 && !mbar_wait(smem_u32(&accempty[ab]), ((it_n >> 1) - 1) & 1, limit,
                                            bp.status)) {
                    flag_error(bp.status, ST_TIMEOUT_MMA);
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)ab * ACC_STRIDE;
                for (int u = 0; u < it.np * SUB; ++u, ++gu) {
                    const int s = gu % UST;
                    if (!mbar_wait(smem_u32(&ufull[s]), (gu / UST) & 1, limit, bp.status)) {
                        flag_error(bp.status, ST_TIMEOUT_UNPACK);
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
                release_item(qi);
            }
            tc_commit_pair(smem_u32(mma_done), BOTH);
        }
    } else if (warp < FIRST_EPI_WARP) {
        // --------------------------------------------------------- unpack --
        // group g takes sub-stage g of every packed stage
        const int grp = (warp - FIRST_UNPACK_WARP) / (UNPACK_WARPS / 2);
        const int wt = ((warp - FIRST_UNPACK_WARP) % (UNPACK_WARPS / 2)) * 32 + lane;
        mxf4rows::RowTask task[TASKS];
#pragma unroll
        for (int j = 0; j < TASKS; ++j)   // over 128 A + 120 B rows
            task[j] = mxf4rows::make_task<HM>(wt + j * GROUP_THREADS, NROWS);
        int gp = 0;
        bool ok = true;
        for (int qi = 0; ok; ++qi) {
            const bool got_item = wait_item(qi);
            if (!__all_sync(0xffffffffu, got_item)) {
                if (lane == 0) flag_error(bp.status, ST_TIMEOUT_FULL);
                break;
            }
            const Item it = items[qi % QSLOTS];
            if (it.job < 0) break;
            for (int kp = 0; kp < it.np; ++kp, ++gp) {
                const int ps = gp % PST;
                const bool got = mbar_wait(smem_u32(&pfull[ps]), (gp / PST) & 1, limit, bp.status);
                if (!__all_sync(0xffffffffu, got)) {
                    if (lane == 0) flag_error(bp.status, ST_TIMEOUT_FULL);
                    ok = false;
                    break;
                }
                const int gu = gp * SUB + grp;
                const int us = gu % UST;
                const bool freed = gu < UST || mbar_wait(smem_u32(&uempty[us]),
                                                         ((gu / UST) - 1) & 1, limit, bp.status);
                if (!__all_sync(0xffffffffu, freed)) {
                    if (lane == 0) flag_error(bp.status, ST_TIMEOUT_MMA);
                    ok = false;
                    break;
                }
                const uint8_t *pa = smem + L::OFF_PA + ps * PA_BYTES;
                const uint8_t *pb = smem + L::OFF_PB + ps * PB_BYTES;
                uint8_t *ua = smem + L::OFF_UA + us * UA_BYTES;
                uint8_t *ub = smem + L::OFF_UB + us * UB_BYTES;
                mxf4rows::unpack_rows(task, pa, pb, ua, ub, grp);
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive_rank(smem_u32(&ufull[us]), 0);
                    mbar_arrive(smem_u32(&pempty[ps]));
                }
            }
            __syncwarp();
            if (lane == 0) release_item(qi);
        }
    } else {
        // ------------------------------------------------------- epilogue --
        // The epilogue warps meet at named barriers, so they must leave the
        // loop together: a failure is recorded in a shared flag that is only
        // read right after the first barrier of an item (every write to it
        // happens before that barrier or between the second and third).
        volatile int *epi_fail = reinterpret_cast<volatile int *>(smem + L::OFF_TMEM + 8);
        const int et = tid - FIRST_EPI_WARP * 32;
        const int ew = warp - FIRST_EPI_WARP;
        const int q = warp & 3;             // TMEM lane quarter
        const int colh = ew >> 2;           // chunks colh, colh + EPI_WARPS / 4, ...
        if (et == 0) *epi_fail = 0;
        named_bar_sync(1, R::EPI_THREADS);
        for (int qi = 0;; ++qi) {
            const bool got_item = wait_item(qi);
            if (!__all_sync(0xffffffffu, got_item) && lane == 0) {
                flag_error(bp.status, ST_TIMEOUT_FULL);
                *epi_fail = 1;
            }
            const Item it = items[qi % QSLOTS];
            named_bar_sync(1, R::EPI_THREADS);
            if (*epi_fail || it.job < 0) break;
            const BatchJob &J = bp.jobs[it.job];
            const int ab = qi & 1;
            if (et < COLS_N) {   // every column factor the chunks read; 0 past the tile and the task
                const int b = it.tb * BN + et;
                const uint32_t cb = (et < BN && b < J.n) ? J.bcB[b] : 0u;
                if constexpr (MODE == R2_EXACT)
                    epi::store_col_f32(colsf, et, cb, J.S);
                else
                    epi::store_col_ref(colsr, et, cb, J.S);
            }
            named_bar_sync(1, R::EPI_THREADS);
            bool ready = mbar_wait(smem_u32(&accfull[ab]), (qi >> 1) & 1, limit, bp.status);
            ready = __all_sync(0xffffffffu, ready);
            if (!ready) {
                if (lane == 0) {
                    flag_error(bp.status, ST_TIMEOUT_MMA);
                    *epi_fail = 1;
                }
            } else {
                __syncwarp();
                tc_fence_after();
                const int a = it.ta * BM + (int)rank * HM + q * 32 + lane;
                const bool a_ok = a < J.m;
                const uint32_t ca = a_ok ? J.bcA[a] : 0u;
                const epi::ARowR ra = epi::make_arow_ref(ca, J.S);
                const epi::ARowF raf = epi::make_arow_f32(ca, J.S);
                const uint32_t tbase =
                    tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)ab * ACC_STRIDE;
                // columns of the last 32-column chunk past the tile's 240 B rows
                // are read but not written
                const int n_tile = it.tb * BN + BN < J.n ? it.tb * BN + BN : J.n;
                const int dlo = diag_lo(J.symmetric, 0), dhi = diag_hi(0);
                epi::SumAcc acc;
                // chunks of CW columns: 32 in exact mode; 16 in reference mode, whose
                // longer epilogue runs faster on fewer live registers (182 against
                // 199 ms on the 4,096-task mix; exact mode: 70.5 against 71.7 ms)
                constexpr int CW = MODE == R2_EXACT ? 32 : 16;
#pragma unroll 1
                for (int c = colh; c < (BN + CW - 1) / CW; c += R::EPI_WARPS / 4) {   // the tile's chunks
                    uint32_t v[CW];
                    __syncwarp();
                    tc_ld_32x32b<CW>(tbase + (uint32_t)(c * CW), v);
                    if constexpr (MODE == R2_EXACT) {
                        epi::chunk_f32<CW>(v, tbase + (uint32_t)(c * CW), raf, colsf, c * CW,
                                           it.tb * BN + c * CW, a, a_ok, n_tile, dlo, dhi, J.r2,
                                           J.ldr, J.counts, J.ldc, 0, J.S);
                        if (J.summary)
                            acc.fold(v, it.tb * BN + c * CW, a, a_ok, J.n, J.symmetric,
                                     J.threshold);
                    } else {
                        // the F32 accumulators hold the counts as floats
                        epi::chunk_ref<0, true, CW>(v, ra, colsr, c * CW, it.tb * BN + c * CW, a,
                                                    a_ok, n_tile, dlo, dhi, J.r2, J.ldr,
                                                    J.counts, J.ldc, 0, J.S);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_rank(smem_u32(&accempty[ab]), 0);
                if (MODE == R2_EXACT && J.summary) acc.flush(J.summary);
            }
            __syncwarp();
            if (lane == 0) release_item(qi);
            named_bar_sync(1, R::EPI_THREADS);   // column factors may be rewritten
        }
    }

    // Teardown: rank 0's last commit arrives on mma_done in both CTAs;
    // neither CTA frees the pair's TMEM or exits while the other may still
    // touch its shared memory.
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        if (!mbar_wait(smem_u32(mma_done), 0, kDrainCycles, nullptr))
            flag_error(bp.status, ST_TIMEOUT_MMA);
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
cudaError_t launch_mode(const BatchParams &bp, int max_ctas, cudaStream_t st) {
    auto kern = k_ld_batch<MODE>;
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
        cfg.blockDim = dim3(Roles<MODE>::THREADS, 1, 1);
        cfg.dynamicSmemBytes = Smem<MODE>::BYTES;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess || n <= 0) {
            (void)cudaGetLastError();
            n = sms / 2;
        }
        g_max_pairs = n;
    }
    long long pairs = bp.nitems < g_max_pairs ? bp.nitems : g_max_pairs;
    if (max_ctas > 0 && 2 * pairs > max_ctas) pairs = max_ctas / 2;
    if (pairs <= 0) return cudaSuccess;
    kern<<<(int)(2 * pairs), Roles<MODE>::THREADS, Smem<MODE>::BYTES, st>>>(bp);
    return cudaGetLastError();
}

}  // namespace

const KernelShape kBatchShape = {BM, BN, PW, HM, HN, 64};
const int kBatchMaxSamples = 1 << 24;

cudaError_t launch_batch(const BatchParams &bp, int r2_mode, int max_ctas, cudaStream_t st) {
    return r2_mode == R2_REFERENCE ? launch_mode<R2_REFERENCE>(bp, max_ctas, st)
                                   : launch_mode<R2_EXACT>(bp, max_ctas, st);
}

}  // namespace qld
