// ld_popc.cu -- counts kernel, variant (a): AND + POPC on the CUDA cores.
//
// Computes C[a][b] = sum_k popc(A[a][k] & B[b][k]) for a 128 x 128 output
// tile per CTA (the binary GEMM of qLD's blis_gemm()/bin_gemm_2x2,
// src/correlator/src/gemm_cpu.c:125-341 and
// blis/config/binary_gemm/kernels/3/bin_gemm.c:4-141) and applies the r^2
// epilogue (gemm_cpu.c:343-404) to the tile before it leaves registers.
//
// Structure (one CTA per SM, 9 warps):
//   warp 8      TMA producer: 2-D tiled loads of 128 rows x 16 words (16 KB,
//               128-byte swizzle) of A and of B per stage into a ring of
//               STAGES stages, completion on a per-stage "full" mbarrier.
//   warps 0-7   consumers: 16 x 16 threads, each owning an 8 x 8 block of
//               (A row, B row) pairs -- A rows tx + 16i, B rows ty + 16j --
//               reading 16-byte chunks (two words) of its 8 + 8 rows from the
//               swizzled stage and doing 4 x (LOP3 + POPC) per pair and chunk.
//               A warp's A loads hit 16 rows whose chunks the swizzle spreads
//               over all banks (2 wavefronts per 256 B: conflict-free), its B
//               loads are 2 broadcast rows.  After a stage each warp arrives
//               on the stage's "empty" mbarrier.
// Every wait is bounded (LdParams::timeout_cycles); on expiry the kernel
// records the cause in the status word and returns without writing output.
#include "qld_device.cuh"
#include "qld_kernels.h"

namespace qld {

namespace {

constexpr int BM = 128, BN = 128;   // output tile (A rows x B rows)
constexpr int KC = 16;              // words per row per stage (128 bytes)
constexpr int TILE_BYTES = BM * KC * 8;
constexpr int CONSUMERS = 256;
constexpr int THREADS = CONSUMERS + 32;

template <int MODE, int STAGES>
__global__ void __launch_bounds__(THREADS, 1)
k_ld_popc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
          const LdParams p) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *sA = smem;
    uint8_t *sB = smem + STAGES * TILE_BYTES;
    uint64_t *full = reinterpret_cast<uint64_t *>(sB + STAGES * TILE_BYTES);
    uint64_t *empty = full + STAGES;

    const int ta = blockIdx.x;
    const int tb = p.tb0 + blockIdx.y;
    // Skip tiles with no entry in the diagonal window (single region: a >= b;
    // band: 1 <= a - b <= band).
    const int dlo = p.band > 0 ? 1 : (p.symmetric ? 0 : -2147483647 - 1);
    const int dhi = p.band > 0 ? p.band : 2147483647;
    if ((long long)ta * BM + BM - 1 - (long long)tb * BN < dlo ||
        (long long)ta * BM - ((long long)tb * BN + BN - 1) > dhi)
        return;
    if (grid_failed(p.status)) return;   // an earlier CTA already gave up

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), CONSUMERS / 32);
        }
        fence_barrier_init();
    }
    __syncthreads();

    if (warp == CONSUMERS / 32) {
        // ----------------------------------------------------- producer --
        if (lane == 0) {
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            int issued = 0;
            for (int kc = 0; kc < p.nk; ++kc) {
                const int s = kc % STAGES;
                if (kc >= STAGES &&
                    !mbar_wait(smem_u32(&empty[s]), ((kc / STAGES) - 1) & 1, p.timeout_cycles, p.status)) {
                    flag_error(p.status, ST_TIMEOUT_EMPTY);
                    break;
                }
                const uint32_t fb = smem_u32(&full[s]);
                mbar_arrive_expect_tx(fb, 2 * TILE_BYTES);
                tma_load_2d(smem_u32(sA + s * TILE_BYTES), &tmA, kc * KC, ta * BM, fb);
                tma_load_2d(smem_u32(sB + s * TILE_BYTES), &tmB, kc * KC, tb * BN, fb);
                ++issued;
            }
            // Drain: no copy may still be in flight when the CTA retires, so
            // these waits ignore other CTAs' errors.
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

    // ------------------------------------------------------- consumers --
    const int tx = tid & 15, ty = tid >> 4;
    const int xa = tx & 7, xb = ty & 7;   // 128-byte swizzle phase of my rows
    uint32_t acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0u;

    for (int kc = 0; kc < p.nk; ++kc) {
        const int s = kc % STAGES;
        if (!mbar_wait(smem_u32(&full[s]), (kc / STAGES) & 1, p.timeout_cycles, p.status)) {
            flag_error(p.status, ST_TIMEOUT_FULL);
            return;
        }
        const uint8_t *a_base = sA + s * TILE_BYTES + tx * 128;
        const uint8_t *b_base = sB + s * TILE_BYTES + ty * 128;
#pragma unroll 1
        for (int c = 0; c < 8; ++c) {
            uint4 av[8], bv[8];
            const int oa = (c ^ xa) << 4, ob = (c ^ xb) << 4;
#pragma unroll
            for (int i = 0; i < 8; ++i)
                av[i] = *reinterpret_cast<const uint4 *>(a_base + i * 16 * 128 + oa);
#pragma unroll
            for (int j = 0; j < 8; ++j)
                bv[j] = *reinterpret_cast<const uint4 *>(b_base + j * 16 * 128 + ob);
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    acc[i][j] += (__popc(av[i].x & bv[j].x) + __popc(av[i].y & bv[j].y)) +
                                 (__popc(av[i].z & bv[j].z) + __popc(av[i].w & bv[j].w));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&empty[s]));
    }

    // -------------------------------------------------------- epilogue --
    const int a0 = ta * BM + tx, b0 = tb * BN + ty;
    if (MODE == R2_EXACT) {
        RowExact ra[8], rb[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) ra[i] = row_exact(a0 + 16 * i < p.m ? p.bcA[a0 + 16 * i] : 0u, p.S);
#pragma unroll
        for (int j = 0; j < 8; ++j) rb[j] = row_exact(b0 + 16 * j < p.n ? p.bcB[b0 + 16 * j] : 0u, p.S);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int b = b0 + 16 * j;
            if (b >= p.n) break;
            float *out = p.r2 + (long long)(b - p.out_row0) * p.ldr;
            uint32_t *cnt = p.counts ? p.counts + (long long)(b - p.out_row0) * p.ldc : nullptr;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int a = a0 + 16 * i;
                if (a < p.m && a - b >= dlo && a - b <= dhi) {
                    out[a] = r2_exact(acc[i][j], ra[i], rb[j], p.S);
                    if (cnt) cnt[a] = acc[i][j];
                }
            }
        }
    } else {
        RowRef ra[8], rb[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) ra[i] = row_ref(a0 + 16 * i < p.m ? p.bcA[a0 + 16 * i] : 0u, p.S);
#pragma unroll
        for (int j = 0; j < 8; ++j) rb[j] = row_ref(b0 + 16 * j < p.n ? p.bcB[b0 + 16 * j] : 0u, p.S);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int b = b0 + 16 * j;
            if (b >= p.n) break;
            float *out = p.r2 + (long long)(b - p.out_row0) * p.ldr;
            uint32_t *cnt = p.counts ? p.counts + (long long)(b - p.out_row0) * p.ldc : nullptr;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int a = a0 + 16 * i;
                if (a < p.m && a - b >= dlo && a - b <= dhi) {
                    out[a] = r2_reference(acc[i][j], ra[i], rb[j], p.S);
                    if (cnt) cnt[a] = acc[i][j];
                }
            }
        }
    }
}

constexpr int POPC_STAGES = 4;

template <int MODE>
cudaError_t launch_mode(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                        int tiles_b, cudaStream_t st) {
    const size_t smem = 1024 + 2 * POPC_STAGES * TILE_BYTES + 2 * POPC_STAGES * sizeof(uint64_t);
    auto kern = k_ld_popc<MODE, POPC_STAGES>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((p.m + BM - 1) / BM, tiles_b);
    kern<<<grid, THREADS, smem, st>>>(tmA, tmB, p);
    return cudaGetLastError();
}

}  // namespace

const KernelShape kPopcShape = {BM, BN, KC, BM, BN, 128};

cudaError_t launch_popc(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                        int tiles_b, int r2_mode, cudaStream_t st) {
    if (tiles_b <= 0 || p.m <= 0) return cudaSuccess;
    return r2_mode == R2_REFERENCE ? launch_mode<R2_REFERENCE>(tmA, tmB, p, tiles_b, st)
                                   : launch_mode<R2_EXACT>(tmA, tmB, p, tiles_b, st);
}

}  // namespace qld
