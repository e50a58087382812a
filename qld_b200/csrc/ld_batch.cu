// ld_batch.cu -- many independent LD tasks (region pairs of uneven SNP and
// sample counts) in one persistent launch fed by a device work queue.
//
// Per-task arithmetic is that of ld_mma.cu (128 x 256 output tiles, bits
// unpacked to {0, 0x80} bytes, tcgen05.mma.kind::i8 into s32 TMEM
// accumulators holding 2^14 * count, fused r^2 epilogue of qLD
// gemm_cpu.c:343-404); qLD itself runs such task lists one task at a time
// (-inputList, src/correlator/src/input_list.c:205-323 and
// correlate_function.c:59-83).  Here every output tile of every task is a
// work item.  The device job table holds per task its tensor maps, sizes and
// output, and the item prefix offsets; items are numbered task by task
// (tasks sorted by cost on the host, most expensive first).
//
// Work queue: the producer thread of each CTA claims the next item with an
// atomic ticket on a global counter, decodes it into (task, A tile, B tile),
// pushes it into a 4-slot item ring in shared memory, and streams its packed
// stages.  The MMA thread, the unpack warps and the epilogue warps pop the
// same items in the same order; each of them releases a ring slot when done
// with its item.  A ticket past the last item pushes an end marker.
#include "epilogue.cuh"
#include "qld_kernels.h"
#include "tcgen05.cuh"

namespace qld {

namespace {

using namespace tc;

constexpr int BM = 128, BN = 256;
constexpr int PW = 8;
constexpr int SUB = PW / 2;
constexpr int PST = 3;
constexpr int UST = 3;
constexpr int PA_BYTES = BM * PW * 8;
constexpr int PB_BYTES = BN * PW * 8;
constexpr int UA_BYTES = BM * 128;
constexpr int UB_BYTES = BN * 128;
constexpr int UNPACK_WARPS = 12;
constexpr int UNPACK_THREADS = UNPACK_WARPS * 32;
constexpr int EPI_WARPS = 4;
constexpr int EPI_THREADS = EPI_WARPS * 32;
constexpr int FIRST_UNPACK_WARP = 2;
constexpr int FIRST_EPI_WARP = FIRST_UNPACK_WARP + UNPACK_WARPS;
constexpr int THREADS = (FIRST_EPI_WARP + EPI_WARPS) * 32;   // 576
constexpr int TASKS = 2 * (BM + BN) / UNPACK_THREADS;
static_assert(TASKS * UNPACK_THREADS == 2 * (BM + BN), "unpack tasks must divide evenly");
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t IDESC = idesc_i8(BM, BN);
constexpr int QSLOTS = 4;                                    // item ring depth
constexpr int ITEM_USERS = 1 + UNPACK_WARPS + EPI_WARPS;     // arrivals freeing a slot

constexpr int OFF_UA = 0;
constexpr int OFF_UB = OFF_UA + UST * UA_BYTES;
constexpr int OFF_PA = OFF_UB + UST * UB_BYTES;
constexpr int OFF_PB = OFF_PA + PST * PA_BYTES;
constexpr int OFF_ROWS = OFF_PB + PST * PB_BYTES;
constexpr int ROWS_BYTES = BN * epi::COL_BYTES;
constexpr int OFF_ITEMS = OFF_ROWS + ROWS_BYTES;
constexpr int OFF_BAR = OFF_ITEMS + QSLOTS * 16;
constexpr int NBARS = 2 * PST + 2 * UST + 2 + 2 + 1 + 2 * QSLOTS;
constexpr int OFF_TMEM = OFF_BAR + NBARS * 8;
constexpr int SMEM_BYTES = OFF_TMEM + 16 + 1024;
static_assert(SMEM_BYTES <= 232448, "shared memory budget");

struct Item {
    int job, ta, tb, np;   // job < 0: end of the queue
};

struct Task {
    uint32_t src, xr, dst, is_a;
    uint32_t chunk_off[4];
    uint32_t pow2[4];
};

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
__global__ void __launch_bounds__(THREADS, 1)
k_ld_batch(const BatchParams bp) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + OFF_BAR);
    uint64_t *pfull = bars, *pempty = bars + PST;
    uint64_t *ufull = bars + 2 * PST, *uempty = bars + 2 * PST + UST;
    uint64_t *accfull = bars + 2 * PST + 2 * UST;
    uint64_t *accempty = accfull + 2;
    uint64_t *mma_done = accempty + 2;
    uint64_t *ifull = mma_done + 1, *iempty = ifull + QSLOTS;
    Item *items = reinterpret_cast<Item *>(smem + OFF_ITEMS);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + OFF_TMEM);
    const epi::Cols cols(smem + OFF_ROWS, BN);

    if (grid_failed(bp.status)) return;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const long long limit = bp.timeout_cycles;

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
        for (int s = 0; s < QSLOTS; ++s) {
            mbar_init(smem_u32(&ifull[s]), 1);
            mbar_init(smem_u32(&iempty[s]), ITEM_USERS);
        }
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
        // --------------------------------------- work queue + TMA producer --
        if (lane == 0) {
            int gp = 0;
            bool ok = true;
            for (int qi = 0;; ++qi) {
                const int slot = qi % QSLOTS;
                if (qi >= QSLOTS && !mbar_wait(smem_u32(&iempty[slot]), ((qi / QSLOTS) - 1) & 1,
                                               limit, bp.status)) {
                    flag_error(bp.status, ST_TIMEOUT_EMPTY);
                    ok = false;
                }
                const long long g =
                    ok ? (long long)atomicAdd(bp.queue, 1ull) : (long long)bp.nitems;
                Item it;
                if (g < bp.nitems) it = decode_item(bp.jobs, bp.njobs, g);
                else it.job = -1, it.ta = it.tb = it.np = 0;
                items[slot] = it;
                mbar_arrive(smem_u32(&ifull[slot]));   // release: the item is visible
                if (it.job < 0) break;
                const BatchJob &J = bp.jobs[it.job];
                for (int kp = 0; kp < it.np; ++kp, ++gp) {
                    const int s = gp % PST;
                    if (gp >= PST && !mbar_wait(smem_u32(&pempty[s]), ((gp / PST) - 1) & 1,
                                                limit, bp.status)) {
                        flag_error(bp.status, ST_TIMEOUT_EMPTY);
                        ok = false;
                        break;
                    }
                    const uint32_t fb = smem_u32(&pfull[s]);
                    mbar_arrive_expect_tx(fb, PA_BYTES + PB_BYTES);
                    tma_load_2d(smem_u32(smem + OFF_PA + s * PA_BYTES), &J.tmA, kp * PW,
                                it.ta * BM, fb);
                    tma_load_2d(smem_u32(smem + OFF_PB + s * PB_BYTES), &J.tmB, kp * PW,
                                it.tb * BN, fb);
                }
            }
            for (int g = gp > PST ? gp - PST : 0; g < gp; ++g)
                if (!mbar_wait(smem_u32(&pfull[g % PST]), (g / PST) & 1, limit, nullptr)) {
                    flag_error(bp.status, ST_TIMEOUT_DRAIN);
                    break;
                }
        }
    } else if (warp == 1) {
        // ----------------------------------------------------- MMA issuer --
        if (lane == 0) {
            int gu = 0, it_n = 0;
            bool ok = true;
            for (int qi = 0; ok; ++qi, ++it_n) {
                const int slot = qi % QSLOTS;
                if (!mbar_wait(smem_u32(&ifull[slot]), (qi / QSLOTS) & 1, limit, bp.status)) {
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
                const uint32_t d = tmem + (uint32_t)(ab * BN);
                for (int u = 0; u < it.np * SUB; ++u, ++gu) {
                    const int s = gu % UST;
                    if (!mbar_wait(smem_u32(&ufull[s]), (gu / UST) & 1, limit, bp.status)) {
                        flag_error(bp.status, ST_TIMEOUT_UNPACK);
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
                tc_commit(smem_u32(&accfull[ab]));
                mbar_arrive(smem_u32(&iempty[slot]));
            }
            tc_commit(smem_u32(mma_done));
        }
    } else if (warp < FIRST_EPI_WARP) {
        // --------------------------------------------------------- unpack --
        const int ut = tid - FIRST_UNPACK_WARP * 32;
        Task task[TASKS];
#pragma unroll
        for (int j = 0; j < TASKS; ++j) {
            const int t = ut + j * UNPACK_THREADS;
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
        for (int qi = 0; ok; ++qi) {
            const int slot = qi % QSLOTS;
            const bool got_item =
                mbar_wait(smem_u32(&ifull[slot]), (qi / QSLOTS) & 1, limit, bp.status);
            if (!__all_sync(0xffffffffu, got_item)) {
                if (lane == 0) flag_error(bp.status, ST_TIMEOUT_FULL);
                break;
            }
            const Item it = items[slot];
            if (it.job < 0) break;
            for (int kp = 0; kp < it.np && ok; ++kp, ++gp) {
                const int ps = gp % PST;
                const bool got = mbar_wait(smem_u32(&pfull[ps]), (gp / PST) & 1, limit, bp.status);
                if (!__all_sync(0xffffffffu, got)) {
                    if (lane == 0) flag_error(bp.status, ST_TIMEOUT_FULL);
                    ok = false;
                    break;
                }
                const uint8_t *pa = smem + OFF_PA + ps * PA_BYTES;
                const uint8_t *pb = smem + OFF_PB + ps * PB_BYTES;
                for (int sub = 0; sub < SUB; ++sub, ++gu) {
                    const int us = gu % UST;
                    const bool freed = gu < UST || mbar_wait(smem_u32(&uempty[us]),
                                                             ((gu / UST) - 1) & 1, limit,
                                                             bp.status);
                    if (!__all_sync(0xffffffffu, freed)) {
                        if (lane == 0) flag_error(bp.status, ST_TIMEOUT_MMA);
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
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&iempty[slot]));
        }
    } else {
        // ------------------------------------------------------- epilogue --
        // The four epilogue warps meet at named barriers, so they must leave
        // the loop together: a failure is recorded in a shared flag that is
        // only read right after the first barrier of an item (every write to
        // it happens before that barrier or between the second and third).
        volatile int *epi_fail = reinterpret_cast<volatile int *>(smem + OFF_TMEM + 8);
        const int et = tid - FIRST_EPI_WARP * 32;
        const int q = warp & 3;
        if (et == 0) *epi_fail = 0;
        named_bar_sync(1, EPI_THREADS);
        for (int qi = 0;; ++qi) {
            const int slot = qi % QSLOTS;
            const bool got_item =
                mbar_wait(smem_u32(&ifull[slot]), (qi / QSLOTS) & 1, limit, bp.status);
            if (!__all_sync(0xffffffffu, got_item) && lane == 0) {
                flag_error(bp.status, ST_TIMEOUT_FULL);
                *epi_fail = 1;
            }
            const Item it = items[slot];
            named_bar_sync(1, EPI_THREADS);
            if (*epi_fail || it.job < 0) break;
            const BatchJob &J = bp.jobs[it.job];
            const int ab = qi & 1;
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int bl = et + k * EPI_THREADS;
                const int b = it.tb * BN + bl;
                epi::store_col<MODE>(cols, bl, b < J.n ? J.bcB[b] : 0u, J.S);
            }
            named_bar_sync(1, EPI_THREADS);
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
                const int a = it.ta * BM + q * 32 + lane;
                const bool a_ok = a < J.m;
                const epi::ARow ra = epi::make_arow<MODE>(a_ok ? J.bcA[a] : 0u, J.S);
                const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * BN);
#pragma unroll 1
                for (int col0 = 0; col0 < BN; col0 += 32) {
                    uint32_t v[32];
                    __syncwarp();
                    tc_ld_32x32b_x32(tbase + (uint32_t)col0, v);
                    epi::chunk<MODE, COUNT_SHIFT>(v, ra, cols, col0, it.tb * BN + col0, a, a_ok,
                                                  J.n, diag_lo(J.symmetric, 0), diag_hi(0), J.r2,
                                                  J.ldr, J.counts, J.ldc, 0, J.S);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&accempty[ab]));
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&iempty[slot]));
            named_bar_sync(1, EPI_THREADS);   // row factors may be rewritten
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        if (!mbar_wait(smem_u32(mma_done), 0, limit, nullptr))
            flag_error(bp.status, ST_TIMEOUT_MMA);
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(TMEM_COLS)
                     : "memory");
    }
}

int g_sm_count = 0;

template <int MODE>
cudaError_t launch_mode(const BatchParams &bp, int max_ctas, cudaStream_t st) {
    auto kern = k_ld_batch<MODE>;
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
    long long grid = bp.nitems < g_sm_count ? bp.nitems : g_sm_count;
    if (max_ctas > 0 && grid > max_ctas) grid = max_ctas;
    if (grid <= 0) return cudaSuccess;
    kern<<<(int)grid, THREADS, SMEM_BYTES, st>>>(bp);
    return cudaGetLastError();
}

}  // namespace

const KernelShape kBatchShape = {BM, BN, PW, BM, BN, 64};

cudaError_t launch_batch(const BatchParams &bp, int r2_mode, int max_ctas, cudaStream_t st) {
    return r2_mode == R2_REFERENCE ? launch_mode<R2_REFERENCE>(bp, max_ctas, st)
                                   : launch_mode<R2_EXACT>(bp, max_ctas, st);
}

}  // namespace qld
