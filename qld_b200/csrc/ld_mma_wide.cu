// ld_mma_wide.cu -- counts kernel, variant (b) with 256 x 256 output tiles.
//
// Same arithmetic as ld_mma.cu (bits unpacked to {0, 0x80} bytes in shared
// memory, tcgen05.mma.kind::i8 with s32 accumulators in TMEM, accumulators
// hold 2^14 * count, r^2 epilogue of qLD gemm_cpu.c:343-404 on the way out),
// but a CTA tile covers 256 A rows x 256 B rows as two 128 x 256
// accumulators that share every unpacked B stage.  Per multiply-accumulate
// this unpacks 2/3 of the bytes the 128 x 256 tile needs -- the unpack, not
// the tensor pipe, bounds the 128 x 256 kernel -- at the price of a single
// accumulator set (both 256-column accumulators fill the 512 TMEM columns),
// so a tile's epilogue is not overlapped with the next tile's MMAs.
//
// Warp roles (persistent, one CTA per SM, B-tile-row-first tile order):
//   warp 0       TMA producer (8 words = 512 samples of 256 A + 256 B rows
//                per packed stage, 64-byte swizzle).
//   warp 1       TMEM owner (512 columns) and MMA issuer: per unpacked stage
//                (128 samples) 2 x 4 MMAs of 128 x 256 x 32.
//   warps 2-17   workers: unpack every stage of the current tile, then the
//                first UST stages of the next tile, then the epilogue of the
//                current tile (warp w reads TMEM lane quarter w % 4; the four
//                warps of a quarter split the 2 accumulators x 2 column
//                halves), then release the accumulators.
#include "epilogue.cuh"
#include "qld_kernels.h"
#include "tcgen05.cuh"

namespace qld {

namespace {

using namespace tc;

constexpr int BM = 256, BN = 256, HM = 128;   // tile; HM = rows per accumulator
constexpr int PW = 8;                    // packed words per row per packed stage
constexpr int SUB = PW / 2;              // unpacked stages (128 samples) per packed stage
constexpr int PST = 2;                   // packed ring depth
constexpr int UST = 2;                   // unpacked ring depth
constexpr int PA_BYTES = BM * PW * 8;    // 16 KB
constexpr int PB_BYTES = BN * PW * 8;    // 16 KB
constexpr int UA_BYTES = BM * 128;       // 32 KB (two 16 KB halves)
constexpr int UB_BYTES = BN * 128;       // 32 KB
constexpr int WORKER_WARPS = 16;
constexpr int WORKERS = WORKER_WARPS * 32;
constexpr int FIRST_WORKER_WARP = 2;
constexpr int THREADS = (FIRST_WORKER_WARP + WORKER_WARPS) * 32;   // 576
constexpr int TASKS = 2 * (BM + BN) / WORKERS;                     // (row, half) per thread
static_assert(TASKS * WORKERS == 2 * (BM + BN), "unpack tasks must divide evenly");
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t IDESC = idesc_i8(HM, BN);

constexpr int OFF_UA = 0;
constexpr int OFF_UB = OFF_UA + UST * UA_BYTES;
constexpr int OFF_PA = OFF_UB + UST * UB_BYTES;
constexpr int OFF_PB = OFF_PA + PST * PA_BYTES;
constexpr int OFF_ROWS = OFF_PB + PST * PB_BYTES;
constexpr int ROWS_BYTES = BN * epi::COL_BYTES;
constexpr int OFF_BAR = OFF_ROWS + ROWS_BYTES;
constexpr int NBARS = 2 * PST + 2 * UST + 2 + 1;
constexpr int OFF_TMEM = OFF_BAR + NBARS * 8;
constexpr int SMEM_BYTES = OFF_TMEM + 16 + 1024;
static_assert(SMEM_BYTES <= 232448, "shared memory budget");

struct Task {
    uint32_t src, xr, dst, is_a;
    uint32_t chunk_off[4];
    uint32_t pow2[4];
};

// Unpack one 128-sample stage (sub) of packed stage (pa, pb) into (ua, ub).
__device__ __forceinline__ void unpack_stage(const Task (&task)[TASKS], const uint8_t *pa,
                                             const uint8_t *pb, uint8_t *ua, uint8_t *ub,
                                             int sub) {
    uint4 w[TASKS];
#pragma unroll
    for (int j = 0; j < TASKS; ++j)
        w[j] = *reinterpret_cast<const uint4 *>((task[j].is_a ? pa : pb) + task[j].src +
                                                ((sub ^ task[j].xr) << 4));
#pragma unroll
    for (int j = 0; j < TASKS; ++j) {
        uint8_t *dst = (task[j].is_a ? ua : ub) + task[j].dst;
#pragma unroll
        for (int cc = 0; cc < 4; ++cc)
            *reinterpret_cast<uint4 *>(dst + task[j].chunk_off[cc]) =
                unpack_chunk(w[j], task[j].pow2[cc]);
    }
}

template <int MODE>
__global__ void __launch_bounds__(THREADS, 1)
k_ld_mma_wide(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              const LdParams p, const int tiles_b) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + OFF_BAR);
    uint64_t *pfull = bars, *pempty = bars + PST;
    uint64_t *ufull = bars + 2 * PST, *uempty = bars + 2 * PST + UST;
    uint64_t *accfull = bars + 2 * PST + 2 * UST;
    uint64_t *accempty = accfull + 1;
    uint64_t *mma_done = accempty + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + OFF_TMEM);
    const epi::Cols cols(smem + OFF_ROWS, BN);

    if (grid_failed(p.status)) return;
    const TileList<BM, BN> tl{(p.m + BM - 1) / BM, p.tb0, tiles_b, p.symmetric, p.band};
    const int dlo = diag_lo(p.symmetric, p.band), dhi = diag_hi(p.band);
    const int ntiles = tl.count();
    if ((int)blockIdx.x >= ntiles) return;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int np = (p.K + PW - 1) / PW;
    const int nu = np * SUB;                 // unpacked stages per tile

    if (tid == 0) {
        for (int s = 0; s < PST; ++s) {
            mbar_init(smem_u32(&pfull[s]), 1);
            mbar_init(smem_u32(&pempty[s]), WORKER_WARPS);
        }
        for (int s = 0; s < UST; ++s) {
            mbar_init(smem_u32(&ufull[s]), WORKER_WARPS);
            mbar_init(smem_u32(&uempty[s]), 1);
        }
        mbar_init(smem_u32(accfull), 1);
        mbar_init(smem_u32(accempty), WORKER_WARPS);
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
            int gp = 0;
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
                if (it >= 1 && !mbar_wait(smem_u32(accempty), (it - 1) & 1, p.timeout_cycles,
                                          p.status)) {
                    flag_error(p.status, ST_TIMEOUT_MMA);
                    break;
                }
                tc_fence_after();
                for (int u = 0; u < nu; ++u, ++gu) {
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
                    for (int kk = 0; kk < 4; ++kk) {
                        const uint64_t bd = sw128_desc(b0 + kk * 32);
                        const uint32_t acc = (u > 0 || kk > 0) ? 1u : 0u;
                        tc_mma_i8(tmem, sw128_desc(a0 + kk * 32), bd, IDESC, acc);
                        tc_mma_i8(tmem + BN, sw128_desc(a0 + HM * 128 + kk * 32), bd, IDESC, acc);
                    }
                    tc_commit(smem_u32(&uempty[s]));
                }
                tc_commit(smem_u32(accfull));
            }
            tc_commit(smem_u32(mma_done));
        }
    } else {
        // -------------------------------------------------------- workers --
        const int wt = tid - FIRST_WORKER_WARP * 32;
        const int wi = warp - FIRST_WORKER_WARP;
        Task task[TASKS];
#pragma unroll
        for (int j = 0; j < TASKS; ++j) {
            const int t = wt + j * WORKERS;      // (row, half) over 256 A + 256 B rows
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
        // Unpacked-stage stream: stage g belongs to tile g / nu.  `done`
        // counts stages this warp has unpacked; stages of a packed stage are
        // unpacked together when the packed stage is consumed.
        int gu = 0;            // next unpacked stage to produce
        bool ok = true, failed = false;
        const int my_tiles = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
        const int total_u = my_tiles * nu;
        // Produce unpacked stages up to (not including) `limit`.
        auto produce_until = [&](int limit) {
            while (ok && gu < limit) {
                const int gp = gu / SUB;             // packed stage holding stage gu
                const int sub = gu % SUB;
                const int ps = gp % PST;
                if (sub == 0) {
                    const bool got = mbar_wait(smem_u32(&pfull[ps]), (gp / PST) & 1,
                                               p.timeout_cycles, p.status);
                    if (!__all_sync(0xffffffffu, got)) {
                        if (lane == 0) flag_error(p.status, ST_TIMEOUT_FULL);
                        ok = false;
                        break;
                    }
                }
                const int us = gu % UST;
                const bool freed = gu < UST || mbar_wait(smem_u32(&uempty[us]),
                                                         ((gu / UST) - 1) & 1, p.timeout_cycles,
                                                         p.status);
                if (!__all_sync(0xffffffffu, freed)) {
                    if (lane == 0) flag_error(p.status, ST_TIMEOUT_MMA);
                    ok = false;
                    break;
                }
                unpack_stage(task, smem + OFF_PA + ps * PA_BYTES, smem + OFF_PB + ps * PB_BYTES,
                             smem + OFF_UA + us * UA_BYTES, smem + OFF_UB + us * UB_BYTES, sub);
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(smem_u32(&ufull[us]));
                    if (sub == SUB - 1) mbar_arrive(smem_u32(&pempty[ps]));
                }
                ++gu;
            }
        };
        const int q = warp & 3;                 // TMEM lane quarter
        const int acc_i = (wi >> 2) & 1;        // which accumulator (A row half)
        const int colh = wi >> 3;               // which 128-column half
        int it = 0;
        int cur_t = 0, cur_base = 0;   // decode_from: tiles in increasing order
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            int ta, tb;
            tl.decode_from(tile, ta, tb, cur_t, cur_base);
            // this tile's stages, then the next tile's first UST stages
            const int lim = (it + 1) * nu + UST;
            produce_until(lim < total_u ? lim : total_u);
            // B-row factors of this tile (256 of them, threads 0..255)
            if (wt < BN) {
                const int b = tb * BN + wt;
                epi::store_col<MODE>(cols, wt, b < p.n ? p.bcB[b] : 0u, p.S);
            }
            named_bar_sync(1, WORKERS);
            bool ready = ok && !failed && mbar_wait(smem_u32(accfull), it & 1, p.timeout_cycles,
                                                    p.status);
            ready = __all_sync(0xffffffffu, ready);
            if (!ready && !failed) {
                if (lane == 0) flag_error(p.status, ST_TIMEOUT_MMA);
                failed = true;
            }
            if (ready) {
                __syncwarp();
                tc_fence_after();
                const int a = ta * BM + acc_i * HM + q * 32 + lane;
                const bool a_ok = a < p.m;
                const epi::ARow ra = epi::make_arow<MODE>(a_ok ? p.bcA[a] : 0u, p.S);
                const uint32_t tbase =
                    tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc_i * BN + colh * 128);
#pragma unroll 1
                for (int c0 = 0; c0 < 128; c0 += 32) {
                    uint32_t v[32];
                    __syncwarp();
                    tc_ld_32x32b_x32(tbase + (uint32_t)c0, v);
                    epi::chunk<MODE, COUNT_SHIFT>(v, ra, cols, colh * 128 + c0,
                                                  tb * BN + colh * 128 + c0, a, a_ok, p.n,
                                                  dlo, dhi, p.r2, p.ldr, p.counts, p.ldc,
                                                  p.out_row0, p.S);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(accempty));
            }
            named_bar_sync(1, WORKERS);   // row factors may be rewritten
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
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
    auto kern = k_ld_mma_wide<MODE>;
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

const KernelShape kMmaWideShape = {BM, BN, PW, BM, BN, 64};

cudaError_t launch_mma_wide(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                            int tiles_b, int r2_mode, cudaStream_t st) {
    if (tiles_b <= 0 || p.m <= 0) return cudaSuccess;
    return r2_mode == R2_REFERENCE ? launch_mode<R2_REFERENCE>(tmA, tmB, p, tiles_b, st)
                                   : launch_mode<R2_EXACT>(tmA, tmB, p, tiles_b, st);
}

}  // namespace qld
