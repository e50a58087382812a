// tcgen05.cuh -- building blocks of the tensor-core counts kernels:
// UMMA shared-memory descriptors, tcgen05 wrappers, the bit -> byte unpack
// and the static tile list of a launch.
#pragma once

#include "qld_device.cuh"

namespace qld {
namespace tc {

// Instruction descriptor, kind::i8: D = s32 (bits 4-5 = 2), A and B unsigned
// 8-bit (bits 7-9, 10-12 = 0), both K-major (bits 15, 16 = 0),
// N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t idesc_i8(int M, int N) {
    return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

constexpr int COUNT_SHIFT = 14;   // log2(0x80 * 0x80): accumulators hold 2^14 * count

// Instruction descriptor, kind::mxf4 (block-scaled 4-bit): B scale-factor
// byte 0 (bits 4-5), A and B E2M1 (bits 7-9, 10-12 = 1), both K-major,
// N >> 3 at bits 17-22, UE8M0 scale factors (bit 23), M >> 4 at bits 24-28,
// A scale-factor byte 0 (bits 29-30), MMA-K 64 (bit 31 = 0); D is F32.
constexpr uint32_t idesc_mxf4(int M, int N) {
    return (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | (1u << 23) |
           ((uint32_t)(M >> 4) << 24);
}

// The same with both operands' scale factors read from byte `sf_byte` (0 or
// 2) of their TMEM columns: an MMA of K = 64 uses two scale bytes per row,
// for its first and second block of 32 elements.
constexpr uint32_t idesc_mxf4_sf(int M, int N, uint32_t sf_byte) {
    return idesc_mxf4(M, N) | (sf_byte << 29) | (sf_byte << 4);
}

// Bit -> E2M1 spread of the 4-bit kernels.  A 32-bit packed word x becomes
// four words t = 0..3 of eight nibbles, nibble n of word t non-zero iff bit
// 4n + t of x is set: the bit kept in place where it is a valid E2M1 code
// (t = 0: 0b0001 = 0.5, t = 1: 0b0010 = 1.0, t = 2: 0b0100 = 2.0) and bit 3
// (the sign) moved down to 2.0, five ALU instructions per word.  Each 16-byte
// chunk of an unpacked row holds one word t of four packed words: 32
// elements, exactly one scale block, whose UE8M0 scale factor (2, 1, 1/2,
// 1/2 for t = 0..3) makes every 1 x 1 product exactly 1.  MMA k-step kk
// covers chunks 2kk and 2kk + 1, i.e. t = 0, 1 for even kk (scale bytes 0-1
// of a column) and t = 2, 3 for odd kk (bytes 2-3).
template <int T>
__device__ __forceinline__ uint32_t spread_e2m1(uint32_t x) {
    if (T == 0) return x & 0x11111111u;
    if (T == 1) return x & 0x22222222u;
    if (T == 2) return x & 0x44444444u;
    return (x >> 1) & 0x44444444u;
}
constexpr uint32_t kSpreadScales = 0x7E7E7F80u;   // bytes 0x80, 0x7F, 0x7E, 0x7E

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

// D += A x B over K = 64 E2M1 elements (32 bytes per row in each operand),
// with the scale factors read from TMEM at sfa / sfb (block of 32 elements).
__device__ __forceinline__ void tc_mma_mxf4(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate, uint32_t sfa,
                                            uint32_t sfb) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%5], [%6], p;\n\t}"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(sfa), "r"(sfb)
        : "memory");
}

// Write one 32-bit value to 16 consecutive TMEM columns of the warp's 32 lanes.
__device__ __forceinline__ void tc_st_32x32b_x16_fill(uint32_t taddr, uint32_t x) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};"
        ::"r"(taddr), "r"(x) : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
        : "memory");
}

// ----------------------------------------------------- CTA-pair (2 SM) forms --
//
// A cluster of two CTAs (ranks 0 and 1) runs one MMA of M = 256 rows: rank r
// holds A rows [128 r, 128 r + 128) and B rows [N/2 r, N/2 r + N/2) in its
// shared memory at the same offsets, and its 128 x N accumulator in its own
// TMEM.  Rank 0 issues the MMAs.

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_id_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_count_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}

// Every thread of both CTAs: shared-memory writes before it are visible to
// the whole cluster after it.
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Arrive on the mbarrier at the same offset in the shared memory of CTA
// `rank`.  The default (release, CTA-scope) semantics suffice for the two
// handshakes that use it: unpacked stages, written by the generic proxy and
// handed to the tensor core after fence.proxy.async, and accumulators read
// by tcgen05.ld before tcgen05.fence::before_thread_sync.  Cluster-scope
// release/acquire on these barriers made the pair kernel twice as slow.
__device__ __forceinline__ void mbar_arrive_rank(uint32_t bar, uint32_t rank) {
    asm volatile(
        "{\n\t.reg .b32 ra;\n\t"
        "mapa.shared::cluster.u32 ra, %0, %1;\n\t"
        "mbarrier.arrive.shared::cluster.b64 _, [ra];\n\t}"
        ::"r"(bar), "r"(rank)
        : "memory");
}

// Hand a 16-byte record to CTA `rank`: store it at the same shared-memory
// offset there, then arrive on that CTA's mbarrier `bar` with cluster-scope
// release, so a waiter there that acquires at cluster scope sees the record.
__device__ __forceinline__ void st_rank_and_arrive(uint32_t dst, int4 v, uint32_t bar,
                                                   uint32_t rank) {
    asm volatile(
        "{\n\t.reg .b32 rd, rb;\n\t"
        "mapa.shared::cluster.u32 rd, %0, %5;\n\t"
        "mapa.shared::cluster.u32 rb, %6, %5;\n\t"
        "st.shared::cluster.v4.u32 [rd], {%1, %2, %3, %4};\n\t"
        "mbarrier.arrive.release.cluster.shared::cluster.b64 _, [rb];\n\t}"
        ::"r"(dst), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(rank), "r"(bar)
        : "memory");
}

// mbar_wait with cluster-scope acquire (pairs with st_rank_and_arrive).
__device__ __forceinline__ bool mbar_wait_acq_cluster(uint32_t bar, uint32_t parity,
                                                      long long limit,
                                                      const unsigned *status) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity), "r"(20000u)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > limit) return false;
        if (status && *((volatile const unsigned *)status) != 0u) return false;
    }
}

__device__ __forceinline__ void tc_mma_mxf4_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                                 uint32_t idesc, uint32_t accumulate,
                                                 uint32_t sfa, uint32_t sfb) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%5], [%6], p;\n\t}"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(sfa), "r"(sfb)
        : "memory");
}

// TMEM allocation by one warp (CG = 1: this CTA; 2: the CTA pair, issued by
// one warp in each CTA), the column base written to shared memory at `slot`;
// then the warp gives up its right to allocate again, so the CTAs waiting
// for an SM's TMEM are not held back.
template <int CG>
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t cols) {
    if constexpr (CG == 2) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                     "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    } else {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                     "r"(cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}

template <int CG>
__device__ __forceinline__ void tmem_dealloc(uint32_t tmem, uint32_t cols) {
    if constexpr (CG == 2)
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols)
                     : "memory");
    else
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols)
                     : "memory");
}

// Arrive once on the mbarrier at offset `bar` of every CTA in `mask` when the
// pair MMAs issued so far have completed.
__device__ __forceinline__ void tc_commit_pair(uint32_t bar, uint16_t mask) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
        " [%0], %1;" ::"r"(bar), "h"(mask)
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

__device__ __forceinline__ void tc_ld_32x32b_x16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 16 or 32 consecutive TMEM columns of the warp's lane quarter.
template <int CW>
__device__ __forceinline__ void tc_ld_32x32b(uint32_t taddr, uint32_t (&v)[CW]) {
    static_assert(CW == 16 || CW == 32, "16 or 32 columns");
    if constexpr (CW == 16) tc_ld_32x32b_x16(taddr, v);
    else tc_ld_32x32b_x32(taddr, v);
}

__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ uint32_t imul(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("mul.lo.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}

// chunk = ((w_j << s) & 0x80808080)_j with the shift as a multiply by 2^s.
__device__ __forceinline__ uint4 unpack_chunk(const uint4 &w, uint32_t pow2) {
    const uint32_t M = 0x80808080u;
    return make_uint4(imul(w.x, pow2) & M, imul(w.y, pow2) & M, imul(w.z, pow2) & M,
                      imul(w.w, pow2) & M);
}

// One unpack task: half of one packed row (4 of its 8 output chunks).
struct UnpackTask {
    uint32_t src;        // smem offset of the row in a packed stage (before stage base)
    uint32_t xr;         // 64-byte swizzle phase of the packed row
    uint32_t dst;        // smem offset of the row in an unpacked stage
    uint32_t is_a;
    uint32_t chunk_off[4];
    uint32_t pow2[4];
};

// Tile list of one launch: B tile rows tb in [tb0, tb0 + tiles_b), and in
// each the A tiles ta in [ta_lo(tb), ta_hi(tb)) -- all of them for two
// regions, those reaching the diagonal (a >= b somewhere) for a single
// region, those meeting 1 <= a - b <= band for a band.  Tiles are numbered
// B-tile-row first.  Used on the host to size grids, on the device to decode.
template <int BM, int BN>
struct TileList {
    int TA, tb0, tiles_b, symmetric, band;
    __host__ __device__ __forceinline__ int ta_lo(int tb) const {
        if (band > 0) {
            const long long v = (long long)tb * BN + 2 - BM;
            return v <= 0 ? 0 : (int)((v + BM - 1) / BM);
        }
        return symmetric ? (tb * BN) / BM : 0;
    }
    __host__ __device__ __forceinline__ int ta_hi(int tb) const {
        if (band > 0) {
            const long long h = ((long long)band + (long long)tb * BN + BN - 1) / BM + 1;
            return h < TA ? (int)h : TA;
        }
        return TA;
    }
    __host__ __device__ __forceinline__ int count() const {
        int n = 0;
        for (int t = 0; t < tiles_b; ++t) {
            const int c = ta_hi(tb0 + t) - ta_lo(tb0 + t);
            n += c > 0 ? c : 0;
        }
        return n;
    }
    // decode() for a caller whose indices never decrease (a persistent CTA
    // walking its tiles): the walk over B tiles resumes at (t, base), the B
    // tile and the count of tiles before it where the previous call stopped,
    // so a call costs the B tiles stepped over instead of all of them.
    __host__ __device__ __forceinline__ void decode_from(int idx, int &ta, int &tb, int &t,
                                                         int &base) const {
        for (; t < tiles_b; ++t) {
            const int lo = ta_lo(tb0 + t);
            const int c = ta_hi(tb0 + t) - lo;
            const int cc = c > 0 ? c : 0;
            if (idx < base + cc) {
                ta = lo + idx - base;
                tb = tb0 + t;
                return;
            }
            base += cc;
        }
        ta = tb = -1;
    }
    __host__ __device__ __forceinline__ void decode(int idx, int &ta, int &tb) const {
        for (int t = 0; t < tiles_b; ++t) {
            const int lo = ta_lo(tb0 + t);
            const int c = ta_hi(tb0 + t) - lo;
            if (c > 0 && idx < c) {
                ta = lo + idx;
                tb = tb0 + t;
                return;
            }
            idx -= c > 0 ? c : 0;
        }
        ta = tb = -1;
    }
};

// Diagonal window of the entries a launch produces: dlo <= a - b <= dhi.
__host__ __device__ __forceinline__ int diag_lo(int symmetric, int band) {
    return band > 0 ? 1 : (symmetric ? 0 : -2147483647 - 1);
}
__host__ __device__ __forceinline__ int diag_hi(int band) {
    return band > 0 ? band : 2147483647;
}


}  // namespace tc
}  // namespace qld
