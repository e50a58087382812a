// ld_mxf4.cu -- counts kernel, variant (c): bits as 4-bit floats on the
// block-scaled tensor path (tcgen05.mma.kind::mxf4).
//
// The counts C[a][b] = sum_k popc(A[a][k] & B[b][k]) (qLD's blis_gemm /
// bin_gemm_2x2, src/correlator/src/gemm_cpu.c:125-341) are a dot product of
// 0/1 vectors.  Here every bit becomes an E2M1 element -- zero or one
// power of two, chosen per scale block so the spread is five ALU
// instructions per 32 bits (tcgen05.cuh: spread_e2m1) -- packed two per
// byte, with UE8M0 scale factors that make every 1 x 1 product exactly 1.0;
// tcgen05.mma.kind::mxf4 accumulates them in F32, exact while a count stays
// below 2^24.  Against the kind::i8 kernels this halves the bytes the unpack
// writes per bit (4 bits instead of 8), needs 5 instead of 16 ALU
// instructions per 32 bits, and runs the MMA at the 4-bit rate.  With
// R2_EXACT the epilogue evaluates r^2 in FP32 from the exact F32 counts
// (epilogue.cuh: chunk_f32).
//
// Tile and roles as ld_mma_wide.cu: 256 A rows x 240 B rows per CTA tile as
// two 128 x 240 accumulators sharing every unpacked B stage.  TMEM: the
// accumulators at columns 0 and 256, the scale factors at columns 496-511,
// written once at start and shared by A and B.
//   warp 0       TMA producer: 8 packed words (512 samples) of 256 A + 240 B
//                rows per packed stage, 64-byte swizzle.
//   warp 1       TMEM owner and MMA issuer: per unpacked stage (256 samples)
//                2 x 4 MMAs of 128 x 240 x 64.
//   warps 2-17   workers: unpack (w -> four words of nibbles, nibble n of
//                output word t = bit 4n + t of w, the same permutation of
//                the samples for A and B), then the epilogue: warp w reads
//                TMEM lane quarter w % 4 of one accumulator, 4 of its 8
//                32-column chunks, and applies the r^2 epilogue
//                (gemm_cpu.c:343-404) on the way out.
// Every wait is bounded; on expiry the kernel records the cause in the
// status word and returns.
#include "epilogue.cuh"
#include "qld_kernels.h"
#include "tcgen05.cuh"

namespace qld {

namespace {

using namespace tc;

constexpr int BM = 256, BN = 240, HM = 128;
constexpr int PW = 8;                    // packed words per row per packed stage
constexpr int SUB = 2;                   // unpacked stages (256 samples) per packed stage
constexpr int PST = 2;
constexpr int UST = 2;
constexpr int PA_BYTES = BM * PW * 8;    // 16 KB
constexpr int PB_BYTES = BN * PW * 8;    // 15 KB
constexpr int UA_BYTES = BM * 128;       // 32 KB: 256 E2M1 per row
constexpr int UB_BYTES = BN * 128;       // 30 KB
constexpr int WORKER_WARPS = 16;
constexpr int WORKERS = WORKER_WARPS * 32;
constexpr int FIRST_WORKER_WARP = 2;
constexpr int THREADS = (FIRST_WORKER_WARP + WORKER_WARPS) * 32;   // 576
constexpr int NTASK = 2 * (BM + BN);                               // (row, half) tasks
constexpr int TASKS = (NTASK + WORKERS - 1) / WORKERS;
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t ACC1 = 256;           // TMEM column of accumulator 1
constexpr uint32_t SF_COL = 496;         // 16 columns of scale factors
constexpr uint32_t IDESC_EVEN = idesc_mxf4_sf(HM, BN, 0);   // k-steps 0, 2: scale bytes 0-1
constexpr uint32_t IDESC_ODD = idesc_mxf4_sf(HM, BN, 2);    // k-steps 1, 3: scale bytes 2-3
constexpr int COLS_N = 256;              // epilogue column factors (BN used)

constexpr int OFF_UA = 0;
constexpr int OFF_UB = OFF_UA + UST * UA_BYTES;
constexpr int OFF_PA = OFF_UB + UST * UB_BYTES;
constexpr int OFF_PB = OFF_PA + PST * PA_BYTES;
constexpr int OFF_ROWS = OFF_PB + PST * PB_BYTES;
constexpr int ROWS_BYTES = COLS_N * epi::COLR_BYTES;   // R2_EXACT uses 8 of the 16
constexpr int OFF_BAR = OFF_ROWS + ROWS_BYTES;
constexpr int NBARS = 2 * PST + 2 * UST + 2 + 1;
constexpr int OFF_TMEM = OFF_BAR + NBARS * 8;
constexpr int SMEM_BYTES = OFF_TMEM + 16 + 1024;
static_assert(SMEM_BYTES <= 232448, "shared memory budget");
static_assert(OFF_UB % 1024 == 0 && UB_BYTES % 1024 == 0 && OFF_PA % 1024 == 0 &&
                  OFF_PB % 1024 == 0 && PB_BYTES % 1024 == 0,
              "swizzled stages must start on 1024-byte boundaries");
static_assert(ACC1 + BN <= SF_COL && SF_COL + 16 <= TMEM_COLS, "TMEM map");

struct Task {
    uint32_t src, xr, dst, is_a, valid, half;
    uint32_t chunk_off[4];
};

// Output word t of input word x: bit 4n + t of x to bit 4n + 1 (E2M1 1.0).
__device__ __forceinline__ uint4 spread4(const uint4 &w, int t) {
    switch (t) {
    case 0: return make_uint4(spread_e2m1<0>(w.x), spread_e2m1<0>(w.y), spread_e2m1<0>(w.z), spread_e2m1<0>(w.w));
    case 1: return make_uint4(spread_e2m1<1>(w.x), spread_e2m1<1>(w.y), spread_e2m1<1>(w.z), spread_e2m1<1>(w.w));
    case 2: return make_uint4(spread_e2m1<2>(w.x), spread_e2m1<2>(w.y), spread_e2m1<2>(w.z), spread_e2m1<2>(w.w));
    default: return make_uint4(spread_e2m1<3>(w.x), spread_e2m1<3>(w.y), spread_e2m1<3>(w.z), spread_e2m1<3>(w.w));
    }
}

// Unpack one 256-sample stage (sub) of packed stage (pa, pb) into (ua, ub).
__device__ __forceinline__ void unpack_stage(const Task (&task)[TASKS], const uint8_t *pa,
                                             const uint8_t *pb, uint8_t *ua, uint8_t *ub,
                                             int sub) {
    uint4 w[TASKS];
#pragma unroll
    for (int j = 0; j < TASKS; ++j)
        if (task[j].valid)
            w[j] = *reinterpret_cast<const uint4 *>(
                (task[j].is_a ? pa : pb) + task[j].src +
                ((((uint32_t)sub * 2 + task[j].half) ^ task[j].xr) << 4));
#pragma unroll
    for (int j = 0; j < TASKS; ++j) {
        if (!task[j].valid) continue;
        uint8_t *dst = (task[j].is_a ? ua : ub) + task[j].dst;
#pragma unroll
        for (int cc = 0; cc < 4; ++cc)
            *reinterpret_cast<uint4 *>(dst + task[j].chunk_off[cc]) = spread4(w[j], cc);
    }
}

template <int MODE>
__global__ void __launch_bounds__(THREADS, 1)
k_ld_mxf4(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
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
    const epi::ColsR colsr(smem + OFF_ROWS, COLS_N);   // R2_REFERENCE factors
    const epi::ColsF colsf(smem + OFF_ROWS, COLS_N);   // R2_EXACT: FP32 factors

    if (grid_failed(p.status)) return;
    const TileList<BM, BN> tl{(p.m + BM - 1) / BM, p.tb0, tiles_b, p.symmetric, p.band};
    const int dlo = diag_lo(p.symmetric, p.band), dhi = diag_hi(p.band);
    const int ntiles = tl.count();
    if ((int)blockIdx.x >= ntiles) return;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int np = (p.K + PW - 1) / PW;
    const int nu = np * SUB;

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
    // Scale factors: every column SF_COL.. holds the four UE8M0 scales of the
    // spread (kSpreadScales) in every lane, for A and B alike; the
    // four warps 2-5 cover the four TMEM lane quarters.
    if (warp >= FIRST_WORKER_WARP && warp < FIRST_WORKER_WARP + 4)
        tc_st_32x32b_x16_fill(tmem + ((uint32_t)((warp & 3) * 32) << 16) + SF_COL, kSpreadScales);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

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
            const uint32_t sf = tmem + SF_COL;
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
                        const uint32_t id = (kk & 1) ? IDESC_ODD : IDESC_EVEN;
                        tc_mma_mxf4(tmem, sw128_desc(a0 + kk * 32), bd, id, acc, sf, sf);
                        tc_mma_mxf4(tmem + ACC1, sw128_desc(a0 + HM * 128 + kk * 32), bd, id,
                                    acc, sf, sf);
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
            const int t = wt + j * WORKERS;      // (row, half) over 256 A + 240 B rows
            const int row = t >> 1, half = t & 1;
            const bool isA = row < BM;
            const int r = isA ? row : row - BM;
            task[j].valid = t < NTASK;
            task[j].is_a = isA;
            task[j].half = (uint32_t)half;
            task[j].src = (uint32_t)(r * 64);
            task[j].xr = (uint32_t)((r >> 1) & 3);
            task[j].dst = (uint32_t)(r * 128);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc)
                task[j].chunk_off[cc] = (uint32_t)(((half * 4 + cc) ^ (r & 7)) << 4);
        }
        int gu = 0;
        bool ok = true, failed = false;
        const int my_tiles = (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
        const int total_u = my_tiles * nu;
        auto produce_until = [&](int limit) {
            while (ok && gu < limit) {
                const int gp = gu / SUB;
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
        const int colh = wi >> 3;               // chunks colh, colh + 2, colh + 4, colh + 6
        int it = 0;
        int cur_t = 0, cur_base = 0;   // decode_from: tiles in increasing order
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            int ta, tb;
            tl.decode_from(tile, ta, tb, cur_t, cur_base);
            const int lim = (it + 1) * nu + UST;
            produce_until(lim < total_u ? lim : total_u);
            if (wt < COLS_N) {   // every column factor the chunks read; 0 past the tile
                const int b = tb * BN + wt;
                const uint32_t cb = (wt < BN && b < p.n) ? p.bcB[b] : 0u;
                if constexpr (MODE == R2_EXACT)
                    epi::store_col_f32(colsf, wt, cb, p.S);
                else
                    epi::store_col_ref(colsr, wt, cb, p.S);
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
                const uint32_t ca = a_ok ? p.bcA[a] : 0u;
                const epi::ARowR ra = epi::make_arow_ref(ca, p.S);
                const epi::ARowF raf = epi::make_arow_f32(ca, p.S);
                const uint32_t tbase =
                    tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)acc_i * ACC1;
                // columns past the tile's 240 B rows are read but not written
                const int n_tile = tb * BN + BN < p.n ? tb * BN + BN : p.n;
#pragma unroll 1
                for (int c = colh; c < 8; c += 2) {
                    uint32_t v[32];
                    __syncwarp();
                    tc_ld_32x32b_x32(tbase + (uint32_t)(c * 32), v);
                    if constexpr (MODE == R2_EXACT) {
                        epi::chunk_f32(v, tbase + (uint32_t)(c * 32), raf, colsf, c * 32,
                                       tb * BN + c * 32, a, a_ok, n_tile,
                                       dlo, dhi, p.r2, p.ldr, p.counts, p.ldc, p.out_row0, p.S);
                    } else {
                        // the F32 accumulators hold the counts as floats
                        epi::chunk_ref<0, true>(v, ra, colsr, c * 32, tb * BN + c * 32, a, a_ok,
                                            n_tile, dlo, dhi, p.r2, p.ldr, p.counts, p.ldc,
                                            p.out_row0, p.S);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(accempty));
            }
            named_bar_sync(1, WORKERS);
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
    auto kern = k_ld_mxf4<MODE>;
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

const KernelShape kMxf4Shape = {BM, BN, PW, BM, BN, 64};
const int kMxf4MaxSamples = 1 << 24;

cudaError_t launch_mxf4(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                        int tiles_b, int r2_mode, cudaStream_t st) {
    if (tiles_b <= 0 || p.m <= 0) return cudaSuccess;
    return r2_mode == R2_REFERENCE ? launch_mode<R2_REFERENCE>(tmA, tmB, p, tiles_b, st)
                                   : launch_mode<R2_EXACT>(tmA, tmB, p, tiles_b, st);
}

}  // namespace qld
