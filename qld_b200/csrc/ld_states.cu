// ld_states.cu -- qLD's COUNTSTATES mode on the CUDA cores.
//
// countStates_mode (src/correlator/src/correlate_IO.c:472-516) gives every
// (A row, B row) pair a state value st: st = 0, then for each 64-bit word k
// the states present among the word's 64 bit pairs (bit bitA*2 + bitB) are
// ORed into st and st becomes the popcount of the result; the next word
// starts from that count read as a bit set.  The reference's per-bit loop
// (with its early exit once st == 15, which cannot change the popcount)
// reduces per word to
//     st = popc(st | S_k),  S_k bit 0: ~a & ~b != 0   bit 1: ~a & b != 0
//                           bit 2:  a & ~b != 0   bit 3:  a & b != 0
// so each pair costs a few LOP3s, compares and one POPC per word -- a
// sequential fold over the words, not a contraction, so it stays on the
// CUDA cores.  Every word 0..K-1 counts, the zero tail bits of the last one
// included (they are state 00, as in the reference); words past K do not.
//
// Structure as ld_popc.cu: one CTA per 128 x 128 output tile, a TMA producer
// warp staging 128 rows x 16 words (128-byte swizzle) of A and of B per stage,
// and 8 consumer warps of 16 x 16 threads, each folding an 8 x 8 block of
// pairs (A rows tx + 16i, B rows ty + 16j).  Output: one byte per pair,
// st[(b - out_row0) * lds + a], inside the diagonal window (single region:
// a >= b).  Every wait is bounded; on expiry the kernel records the cause in
// the status word and returns.
#include "qld_device.cuh"
#include "qld_kernels.h"

namespace qld {

namespace {

constexpr int BM = 128, BN = 128;
constexpr int KC = 16;
constexpr int TILE_BYTES = BM * KC * 8;
constexpr int CONSUMERS = 256;
constexpr int THREADS = CONSUMERS + 32;
constexpr int STAGES = 4;

// Joint states present in one 64-bit word pair, given as 32-bit halves.
__device__ __forceinline__ uint32_t word_states(uint32_t alo, uint32_t ahi, uint32_t blo,
                                                uint32_t bhi) {
    const uint32_t s11 = (alo & blo) | (ahi & bhi);
    const uint32_t s10 = (alo & ~blo) | (ahi & ~bhi);
    const uint32_t s01 = (~alo & blo) | (~ahi & bhi);
    const uint32_t s00 = ~(alo | blo) | ~(ahi | bhi);
    return (s00 != 0u ? 1u : 0u) | (s01 != 0u ? 2u : 0u) | (s10 != 0u ? 4u : 0u) |
           (s11 != 0u ? 8u : 0u);
}

__global__ void __launch_bounds__(THREADS, 1)
k_states(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
         const StatesParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *sA = smem;
    uint8_t *sB = smem + STAGES * TILE_BYTES;
    uint64_t *full = reinterpret_cast<uint64_t *>(sB + STAGES * TILE_BYTES);
    uint64_t *empty = full + STAGES;

    const int ta = blockIdx.x;
    const int tb = p.tb0 + blockIdx.y;
    const int dlo = p.symmetric ? 0 : -2147483647 - 1;
    if (p.symmetric && (long long)ta * BM + BM - 1 < (long long)tb * BN) return;
    if (grid_failed(p.status)) return;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int nk = (p.K + KC - 1) / KC;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), CONSUMERS / 32);
        }
        fence_barrier_init();
    }
    __syncthreads();

    if (warp == CONSUMERS / 32) {
        if (lane == 0) {
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            int issued = 0;
            for (int kc = 0; kc < nk; ++kc) {
                const int s = kc % STAGES;
                if (kc >= STAGES && !mbar_wait(smem_u32(&empty[s]), ((kc / STAGES) - 1) & 1,
                                               p.timeout_cycles, p.status)) {
                    flag_error(p.status, ST_TIMEOUT_EMPTY);
                    break;
                }
                const uint32_t fb = smem_u32(&full[s]);
                mbar_arrive_expect_tx(fb, 2 * TILE_BYTES);
                tma_load_2d(smem_u32(sA + s * TILE_BYTES), &tmA, kc * KC, ta * BM, fb);
                tma_load_2d(smem_u32(sB + s * TILE_BYTES), &tmB, kc * KC, tb * BN, fb);
                ++issued;
            }
            for (int kc = issued > STAGES ? issued - STAGES : 0; kc < issued; ++kc) {
                if (!mbar_wait(smem_u32(&full[kc % STAGES]), (kc / STAGES) & 1,
                               kDrainCycles, nullptr)) {
                    flag_error(p.status, ST_TIMEOUT_DRAIN);
                    break;
                }
            }
        }
        return;
    }

    const int tx = tid & 15, ty = tid >> 4;
    const int xa = tx & 7, xb = ty & 7;
    uint32_t st[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) st[i][j] = 0u;

    for (int kc = 0; kc < nk; ++kc) {
        const int s = kc % STAGES;
        if (!mbar_wait(smem_u32(&full[s]), (kc / STAGES) & 1, p.timeout_cycles, p.status)) {
            flag_error(p.status, ST_TIMEOUT_FULL);
            return;
        }
        const int words = p.K - kc * KC < KC ? p.K - kc * KC : KC;   // words past K: skip
        const uint8_t *a_base = sA + s * TILE_BYTES + tx * 128;
        const uint8_t *b_base = sB + s * TILE_BYTES + ty * 128;
#pragma unroll 1
        for (int c = 0; 2 * c < words; ++c) {
            uint4 av[8], bv[8];
            const int oa = (c ^ xa) << 4, ob = (c ^ xb) << 4;
#pragma unroll
            for (int i = 0; i < 8; ++i)
                av[i] = *reinterpret_cast<const uint4 *>(a_base + i * 16 * 128 + oa);
#pragma unroll
            for (int j = 0; j < 8; ++j)
                bv[j] = *reinterpret_cast<const uint4 *>(b_base + j * 16 * 128 + ob);
            const bool second = 2 * c + 1 < words;
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    uint32_t v = __popc(st[i][j] | word_states(av[i].x, av[i].y, bv[j].x, bv[j].y));
                    if (second)
                        v = __popc(v | word_states(av[i].z, av[i].w, bv[j].z, bv[j].w));
                    st[i][j] = v;
                }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&empty[s]));
    }

    const int a0 = ta * BM + tx, b0 = tb * BN + ty;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int b = b0 + 16 * j;
        if (b >= p.n) break;
        uint8_t *out = p.out + (long long)(b - p.out_row0) * p.lds;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int a = a0 + 16 * i;
            if (a < p.m && a - b >= dlo) out[a] = (uint8_t)st[i][j];
        }
    }
}

}  // namespace

const KernelShape kStatesShape = {BM, BN, KC, BM, BN, 128};

cudaError_t launch_states(const CUtensorMap &tmA, const CUtensorMap &tmB, const StatesParams &p,
                          int tiles_b, cudaStream_t st) {
    if (tiles_b <= 0 || p.m <= 0) return cudaSuccess;
    const size_t smem = 1024 + 2 * STAGES * TILE_BYTES + 2 * STAGES * sizeof(uint64_t);
    cudaError_t e =
        cudaFuncSetAttribute(k_states, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((p.m + BM - 1) / BM, tiles_b);
    k_states<<<grid, THREADS, smem, st>>>(tmA, tmB, p);
    return cudaGetLastError();
}

}  // namespace qld
