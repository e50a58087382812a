// vcf_pack.cu -- VCF genotype fields -> packed MDF rows on the GPU: the
// per-sample part of qLD-parse-2MDF (src/mdf_extension/src/process_data.c:
// 152-328 with snip_processing.c:270-427,473-797).
//
// The host hands over the text of each VCF data line that passed the fixed-
// field checks, from its first sample field to the end of the line, and the
// line's GT position and REF/ALT states.  One CTA works on one site:
//   1. Fields: a field starts at a byte that is not a separator (space or
//      tab, as getWordFromString, read_file.c:99-137) right after a
//      separator or at the segment start.  Each thread takes a contiguous
//      byte chunk and owns the fields that start in it; a block prefix of
//      the per-chunk field counts gives every field its sample index.
//   2. Genotype: for a valid sample, the GT subfield as getGTfield leaves it
//      (it copies subfield GT to the front of the field and writes a
//      terminator only if a ':' follows; otherwise the rest of the original
//      field stays behind it), then getGTdata: digits become states[digit],
//      '.' becomes 'N', '|' closes a phased group, '/' extends an unphased
//      one, and an unphased group is shuffled with rand() (dataShuffleKnuth).
//      The sample contributes dataSize = separators + 1 characters.
//   3. A block prefix of the per-chunk character counts places every
//      sample's characters in the site's row (scratch memory).  Unphased
//      groups take their random numbers in sample order from `rnd`, at the
//      site's offset `rnd_off` (the sites' counts come from a first launch
//      that only counts).
//   4. The row: c0 = its first non-N base.  The site is dropped unless a
//      second base appears and no 'N' comes before that first second base
//      (removeNonPolymorphicSiteDNA with its early exit, :532-601).  A kept
//      site has bit 1 for every sample character that is a base other than c0
//      (binaryDeduction + convertAlignmentBIN + compressSnip_x64, :718-797):
//      MSB-first in K words, BC = the number of ones, zero bits past the row.
// Errors are per site codes; the host reports the first failing site in
// file order, as qLD exits on the first one.
#include <cstdint>

#include "qld_kernels.h"

namespace qld {
namespace {

constexpr int THREADS = 256;

__device__ __forceinline__ bool is_sep(char c) { return c == ' ' || c == '\t'; }

// Effective GT string of one field (see 2.): chars [g0, g1) then, when no
// ':' ends the subfield, the field's own chars from (g1 - g0) onward.
struct GtView {
    const char *f;
    int flen, g0, g1;
    bool terminated;
    __device__ __forceinline__ int length() const {
        return (g1 - g0) + (terminated ? 0 : (flen - (g1 - g0)));
    }
    __device__ __forceinline__ char at(int i) const {
        return i < g1 - g0 ? f[g0 + i] : f[i];
    }
};

__device__ GtView gt_view(const char *f, int flen, int gt_pos) {
    GtView v{f, flen, 0, 0, false};
    int pos = gt_pos;
    int i = 0;
    for (; i < flen && pos > 0; ++i)   // skip gt_pos subfields
        if (f[i] == ':') --pos;
    if (pos > 0) return v;             // fewer subfields: nothing copied, the field stays whole
    v.g0 = i;
    for (; i < flen && f[i] != ':'; ++i) {}
    v.g1 = i;
    v.terminated = i < flen;
    return v;
}

struct SampleOut {
    char c[3];
    int n;          // characters getGTdata produced (digits and dots)
    int data_size;  // separators in the copied GT subfield + 1
    int slashes;    // rand() calls its shuffles make
    int err;
};

// getGTdata without the random swaps (they are applied by shuffle_sample).
__device__ SampleOut parse_sample(const char *f, int flen, int gt_pos, const char *states,
                                  int n_states) {
    SampleOut o{{0, 0, 0}, 0, 1, 0, 0};
    const GtView v = gt_view(f, flen, gt_pos);
    if (v.length() <= 0) { o.err = QLD_VCF_EMPTY_GT; return o; }
    for (int i = v.g0; i < v.g1; ++i)
        if (f[i] == '|' || f[i] == '/') ++o.data_size;
    const int L = v.length();
    int start = 0, end = 0;
    for (int i = 0; i < L; ++i) {
        const char ch = v.at(i);
        if (ch >= '0' && ch <= '9') {
            const int idx = ch - '0';
            if (idx >= n_states) { o.err = QLD_VCF_ALLELE; return o; }
            if (o.n + 1 >= 4) { o.err = QLD_VCF_ALLELES; return o; }
            o.c[o.n++] = states[idx];
        } else if (ch == '.') {
            if (o.n + 1 >= 4) { o.err = QLD_VCF_ALLELES; return o; }
            o.c[o.n++] = 'N';
        } else if (ch == '/') {
            ++end;
        } else if (ch == '|') {
            o.slashes += end > start ? end - start : 0;
            start = end = o.n;
        }
    }
    o.slashes += end > start ? end - start : 0;
    return o;
}

// Apply the unphased shuffles of one sample with its random numbers
// (dataShuffleKnuth, snip_processing.c:337-353), re-walking its GT string.
__device__ void shuffle_sample(const char *f, int flen, int gt_pos, SampleOut &o,
                               const unsigned *rnd, long long &r) {
    const GtView v = gt_view(f, flen, gt_pos);
    const int L = v.length();
    int start = 0, end = 0, n = 0;
    auto knuth = [&](int s, int e) {
        for (int i = e; i > s; --i) {
            const int idx = s + (int)(rnd[r++] % (unsigned)(i - s + 1));
            if (idx < 3 && i < 3) {
                const char t = o.c[idx];
                o.c[idx] = o.c[i];
                o.c[i] = t;
            }
        }
    };
    for (int i = 0; i < L; ++i) {
        const char ch = v.at(i);
        if ((ch >= '0' && ch <= '9') || ch == '.') ++n;
        else if (ch == '/') ++end;
        else if (ch == '|') {
            if (end > start) knuth(start, end);
            start = end = n;
        }
    }
    if (end > start) knuth(start, end);
}

// Block-wide exclusive scan of one value per thread; *total receives the sum.
__device__ long long block_scan(long long x, long long *total) {
    __shared__ long long warp_sum[THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long v = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += y;
    }
    if (lane == 31) warp_sum[wid] = v;
    __syncthreads();
    if (wid == 0) {
        long long w = lane < THREADS / 32 ? warp_sum[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w += y;
        }
        if (lane < THREADS / 32) warp_sum[lane] = w;
    }
    __syncthreads();
    const long long before = (wid > 0 ? warp_sum[wid - 1] : 0) + v - x;
    *total = warp_sum[THREADS / 32 - 1];
    __syncthreads();
    return before;
}

__device__ int block_min(int x) {
    __shared__ int red[THREADS / 32];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) x = min(x, __shfl_xor_sync(0xffffffffu, x, d));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    int r = red[0];
#pragma unroll
    for (int w = 1; w < THREADS / 32; ++w) r = min(r, red[w]);
    __syncthreads();
    return r;
}

// Fields starting in [c0, c1) of a segment: fn(field_ptr, field_len) in order.
template <typename F>
__device__ __forceinline__ void for_fields(const char *t, int len, int c0, int c1, F fn) {
    for (int p = c0; p < c1; ++p) {
        if (is_sep(t[p]) || (p > 0 && !is_sep(t[p - 1]))) continue;
        int e = p;
        while (e < len && !is_sep(t[e])) ++e;
        fn(t + p, e - p);
        p = e;   // the separator at e (if any) cannot start a field
    }
}

__global__ void __launch_bounds__(THREADS)
k_vcf_sites(const char *__restrict__ text, const qld_vcf_site *__restrict__ sites, int nsites,
            const uint8_t *__restrict__ valid, int nsamples, int ploidy, int K,
            const unsigned *__restrict__ rnd, const long long *__restrict__ rnd_off,
            long long *__restrict__ slash_count, char *__restrict__ scratch, int scratch_cap,
            uint64_t *__restrict__ words, uint32_t *__restrict__ bc, int *__restrict__ snip_len,
            uint8_t *__restrict__ keep, int *__restrict__ err) {
    const bool pack = rnd_off != nullptr;
    char *row = scratch + (long long)blockIdx.x * scratch_cap;
    for (int s = blockIdx.x; s < nsites; s += gridDim.x) {
        const qld_vcf_site site = sites[s];
        const char *t = text + site.off;
        const int len = site.len;
        const int chunk = (len + THREADS - 1) / THREADS;
        const int c0 = min(len, (int)threadIdx.x * chunk), c1 = min(len, c0 + chunk);
        // 1. fields per chunk -> sample index of my first field
        int nf = 0;
        for_fields(t, len, c0, c1, [&](const char *, int) { ++nf; });
        long long nfields;
        const long long fbase = block_scan(nf, &nfields);
        // 2. characters and rand() calls per chunk
        int nchar = 0, nslash = 0, myerr = 0;
        {
            long long si = fbase;
            for_fields(t, len, c0, c1, [&](const char *f, int flen) {
                const long long sample = si++;
                if (myerr) return;
                if (sample >= nsamples) { myerr = QLD_VCF_SAMPLES; return; }
                if (!valid[sample]) return;
                const SampleOut o = parse_sample(f, flen, site.gt_pos, site.states, site.n_states);
                if (o.err) { myerr = o.err; return; }
                if (o.data_size > ploidy) { myerr = QLD_VCF_PLOIDY; return; }
                if (o.n < o.data_size) { myerr = QLD_VCF_SHORT_GT; return; }
                nchar += o.data_size;
                nslash += o.slashes;
            });
        }
        long long total_chars, total_slash;
        const long long cbase = block_scan(nchar, &total_chars);
        const long long rbase = block_scan(nslash, &total_slash);
        const int first_err = block_min(myerr ? myerr : 0x7fffffff);
        if (!pack) {
            if (threadIdx.x == 0) {
                slash_count[s] = total_slash;
                snip_len[s] = (int)total_chars;
                err[s] = first_err == 0x7fffffff ? 0 : first_err;
            }
            continue;
        }
        if (first_err != 0x7fffffff || total_chars > scratch_cap || total_chars == 0 ||
            total_chars > (long long)K * 64) {
            if (threadIdx.x == 0) {
                err[s] = first_err != 0x7fffffff ? first_err
                         : total_chars == 0      ? QLD_VCF_NO_SAMPLES
                                                 : QLD_VCF_PLOIDY;
                keep[s] = 0;
                snip_len[s] = (int)total_chars;
                bc[s] = 0;
            }
            for (int w = threadIdx.x; w < K; w += THREADS) words[(long long)s * K + w] = 0;
            continue;
        }
        // 3. characters into the row, shuffled with this site's random numbers
        int first_base = 0x7fffffff, first_n = 0x7fffffff;
        {
            long long si = fbase, pos = cbase, r = rnd_off[s] + rbase;
            for_fields(t, len, c0, c1, [&](const char *f, int flen) {
                const long long sample = si++;
                if (!valid[sample]) return;
                SampleOut o = parse_sample(f, flen, site.gt_pos, site.states, site.n_states);
                if (o.slashes) shuffle_sample(f, flen, site.gt_pos, o, rnd, r);
                for (int k = 0; k < o.data_size; ++k) {
                    const char ch = o.c[k];
                    if (ch == 'N') first_n = min(first_n, (int)pos);
                    else first_base = min(first_base, (int)pos);
                    row[pos++] = ch;
                }
            });
        }
        __syncthreads();
        const int p0 = block_min(first_base);
        first_n = block_min(first_n);
        // 4. the second base, validity of the characters
        int second = 0x7fffffff, bad = 0;
        const int L = (int)total_chars;
        const char cb = p0 < L ? row[p0] : 'N';
        for (int i = threadIdx.x; i < L; i += THREADS) {
            const char ch = row[i];
            if (ch != 'A' && ch != 'C' && ch != 'G' && ch != 'T' && ch != 'N') bad = 1;
            else if (ch != 'N' && ch != cb) second = min(second, i);
        }
        second = block_min(second);
        bad = block_min(bad ? 0 : 1) == 0;
        const bool kept = !bad && second < L && first_n > second;
        if (threadIdx.x == 0) {
            snip_len[s] = L;
            keep[s] = kept ? 1 : 0;
            err[s] = bad ? QLD_VCF_STATE_CHAR : 0;
        }
        // bits: a base other than c0
        unsigned ones = 0;
        uint64_t *wrow = words + (long long)s * K;
        for (int w = threadIdx.x; w < K; w += THREADS) {
            uint64_t x = 0;
            if (kept) {
                const int b0 = w * 64;
                for (int k = 0; k < 64; ++k) {
                    const int i = b0 + k;
                    const char ch = i < L ? row[i] : 'N';
                    x = (x << 1) | (uint64_t)(ch != 'N' && ch != cb);
                }
            }
            wrow[w] = x;
            ones += (unsigned)__popcll(x);
        }
        long long total_ones;
        block_scan(ones, &total_ones);
        if (threadIdx.x == 0) bc[s] = (uint32_t)total_ones;
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_vcf_sites(const char *text, const qld_vcf_site *sites, int nsites,
                             const uint8_t *valid, int nsamples, int ploidy, int K,
                             const unsigned *rnd, const long long *rnd_off,
                             long long *slash_count, char *scratch, int scratch_cap, int ctas,
                             uint64_t *words, uint32_t *bc, int *snip_len, uint8_t *keep,
                             int *err, cudaStream_t st) {
    if (nsites <= 0) return cudaSuccess;
    k_vcf_sites<<<ctas, THREADS, 0, st>>>(text, sites, nsites, valid, nsamples, ploidy, K, rnd,
                                         rnd_off, slash_count, scratch, scratch_cap, words, bc,
                                         snip_len, keep, err);
    return cudaGetLastError();
}

}  // namespace qld
