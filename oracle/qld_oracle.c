/*
 * qld_oracle.c -- CPU restatement of qLD-compute's LD hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; nothing in the shipped library links, loads or calls it.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it.
 *
 * What is restated (reference file:line, paths inside the qLD project):
 *   qo_counts          <- blis_gemm() / gemm() + bin_gemm_2x2()
 *                         src/correlator/src/gemm_cpu.c:125-341,
 *                         blis/config/binary_gemm/kernels/3/bin_gemm.c:4-141
 *                         C[a + b*m] = sum_k popcount(A[a*K+k] & B[b*K+k]),
 *                         column-major m x n; the single-region (SYRK, CblasLower)
 *                         form fills only a >= b and leaves the rest 0
 *                         (gemm_cpu.c:226-236 and the zeroing at :479-483).
 *   qo_r2_reference    <- get_pairwise_ld_score()  gemm_cpu.c:343-404, with the
 *                         same float/double mix, written out operation by
 *                         operation so the rounding is explicit.
 *   qo_r2_exact        FP64 oracle: r2 = D^2 / (cA(S-cA) cB(S-cB)) with the exact
 *                         integer D = S*cAB - cA*cB, and the reference's special
 *                         cases (zero popcount -> 0, > 1.0001 -> 123.456).
 *   qo_write_results   <- writeResultsHeader()/writeResults() correlate_IO.c:378-429
 *   qo_fprint_f        <- fprint_f()/reverse()  fast_print.c:21-103
 *   qo_count_states    <- countStates_mode()  correlate_IO.c:472-516 (the
 *                         COUNTSTATES build), bit loop and all
 *   qo_write_states    <- writeStateCount()   correlate_IO.c:430-470
 *   qo_vcf_pack        <- qLD-parse-2MDF's per-site processing: getGTfield,
 *                         getGTdata, determineStates,
 *                         removeNonPolymorphicSite, binaryDeduction,
 *                         compressSnip_x64 (src/mdf_extension/src/
 *                         process_data.c:152-328, snip_processing.c:270-797)
 *
 * Build with -ffp-contract=off: every fused multiply-add below is written as
 * an explicit fmaf() so the rounding never depends on compiler flags.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define QO_EXPORT __attribute__((visibility("default")))

/* ---------------------------------------------------------------- counts -- */

QO_EXPORT void qo_counts(const uint64_t *A, int m, const uint64_t *B, int n,
                         int K, int lower_only, uint32_t *C)
{
#pragma omp parallel for schedule(dynamic, 8)
    for (int b = 0; b < n; b++) {
        const uint64_t *rb = B + (size_t)b * K;
        for (int a = 0; a < m; a++) {
            uint32_t c = 0;
            if (!lower_only || a >= b) {
                const uint64_t *ra = A + (size_t)a * K;
                for (int k = 0; k < K; k++)
                    c += (uint32_t)__builtin_popcountll(ra[k] & rb[k]);
            }
            C[(size_t)a + (size_t)b * m] = c;
        }
    }
}

/* Row popcounts: the MDF "BC" field / BCtable (snip_processing.c:805). */
QO_EXPORT void qo_bitcounts(const uint64_t *A, int m, int K, uint32_t *bc)
{
    for (int a = 0; a < m; a++) {
        uint32_t c = 0;
        for (int k = 0; k < K; k++)
            c += (uint32_t)__builtin_popcountll(A[(size_t)a * K + k]);
        bc[a] = c;
    }
}

/* ------------------------------------------------------------ r2 epilogue -- */

/*
 * get_pairwise_ld_score (gemm_cpu.c:343-404), entry (i over B, j over A):
 *   val_1 = (float)bcA[j] / S; val_2 = (float)bcB[i] / S; val_3 = (float)C / S
 *   r  = (val_3 - val_1*val_2)^2                        (float)
 *   r /= (val_1*val_2*(1.0-val_1)*(1.0-val_2))           (double denominator)
 *   r > 1.0001 -> 123.456
 * `fma_contract` selects whether val_3 - val_1*val_2 is one fused operation
 * (what gcc emits for the reference's -O3 -march=native build on FMA hosts)
 * or a rounded product followed by a rounded subtraction.
 */
static inline float ref_entry(uint32_t cA, uint32_t cB, uint32_t cAB, int S,
                              int fma_contract)
{
    if (cB == 0 || cA == 0)
        return 0.0f;
    float fs = (float)S;
    float v1 = (float)cA / fs;
    float v2 = (float)cB / fs;
    float v3 = (float)cAB / fs;
    float d;
    if (fma_contract) {
        d = fmaf(-v1, v2, v3);
    } else {
        volatile float p = v1 * v2;
        d = v3 - p;
    }
    float r = d * d;
    float p12 = v1 * v2;
    double den = (double)p12 * (1.0 - (double)v1);
    den = den * (1.0 - (double)v2);
    r = (float)((double)r / den);
    if ((double)r > 1.0001)
        r = 123.456f;
    return r;
}

/* out[i*m + j] for i < n (B rows), j < m (A rows); C column-major m x n. */
QO_EXPORT void qo_r2_reference(const uint32_t *bcA, int m, const uint32_t *bcB,
                               int n, const uint32_t *C, int S,
                               int fma_contract, float *out)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++)
        for (int j = 0; j < m; j++)
            out[(size_t)i * m + j] =
                ref_entry(bcA[j], bcB[i], C[(size_t)j + (size_t)i * m], S,
                          fma_contract);
}

static inline double exact_entry(uint32_t cA, uint32_t cB, uint32_t cAB, int S)
{
    if (cB == 0 || cA == 0)
        return 0.0;
    long long D = (long long)S * cAB - (long long)cA * cB;
    long long vA = (long long)cA * ((long long)S - cA);
    long long vB = (long long)cB * ((long long)S - cB);
    long double num = (long double)D * (long double)D;
    long double den = (long double)vA * (long double)vB;
    double r = (double)(num / den);
    if (r > 1.0001)
        r = 123.456;
    return r;
}

/* FP64 oracle; out64 and/or out32 (its float rounding) may be NULL. */
QO_EXPORT void qo_r2_exact(const uint32_t *bcA, int m, const uint32_t *bcB,
                           int n, const uint32_t *C, int S, double *out64,
                           float *out32)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++)
        for (int j = 0; j < m; j++) {
            double r = exact_entry(bcA[j], bcB[i], C[(size_t)j + (size_t)i * m], S);
            if (out64)
                out64[(size_t)i * m + j] = r;
            if (out32)
                out32[(size_t)i * m + j] = (r == 123.456) ? 123.456f : (float)r;
        }
}

/* ------------------------------------------------------------ text report -- */

typedef struct {
    char *buf;
    size_t len, cap;
} qo_sink;

static void sink_putc(qo_sink *s, char c)
{
    if (s->len < s->cap)
        s->buf[s->len] = c;
    s->len++;
}

static void sink_puts(qo_sink *s, const char *str)
{
    while (*str)
        sink_putc(s, *str++);
}

/* reverse() of fast_print.c:21-33: reverses the decimal digits of a positive
 * value in place and returns their count; a value <= 0 becomes 0. */
static unsigned rev_digits(long *num)
{
    unsigned digits = 0;
    long rev = 0;
    while (*num > 0) {
        digits++;
        rev = rev * 10 + (*num) % 10;
        *num /= 10;
    }
    *num = rev;
    return digits;
}

/* fprint_f (fast_print.c:35-103): the scaled value is formed in float and
 * truncated, never rounded; a zero fraction prints as "<int>." */
static void fmt_f(qo_sink *s, float val, int precision)
{
    unsigned long power10 = 1;
    for (int j = 0; j < precision; j++)
        power10 *= 10;
    long scaled = (long)(val * (float)power10);
    long ipart = (long)val;
    scaled = (long)((unsigned long)scaled - (unsigned long)ipart * power10);
    unsigned i_digits = rev_digits(&ipart);
    unsigned d_digits = rev_digits(&scaled);
    if (ipart == 0) {
        sink_putc(s, '0');
    } else {
        unsigned printed = 0;
        while (ipart != 0) {
            sink_putc(s, (char)('0' + ipart % 10));
            ipart /= 10;
            printed++;
        }
        for (unsigned j = 0; j < i_digits - printed; j++)
            sink_putc(s, '0');
    }
    sink_putc(s, '.');
    if (scaled == 0)
        return;
    for (unsigned j = 0; j < (unsigned)precision - d_digits; j++)
        sink_putc(s, '0');
    for (unsigned j = 0; j < d_digits; j++) {
        sink_putc(s, (char)('0' + scaled % 10));
        scaled /= 10;
    }
}

QO_EXPORT size_t qo_fprint_f(char *buf, size_t cap, float val, int precision)
{
    qo_sink s = {buf, 0, cap};
    fmt_f(&s, val, precision);
    return s.len;
}

/*
 * Report body of writeResults (correlate_IO.c:384-429), preceded by the
 * header line of writeResultsHeader (:378-381) when with_header != 0.
 * Returns the number of bytes the report needs; writes at most cap bytes.
 */
QO_EXPORT size_t qo_write_results(char *buf, size_t cap, int with_header,
                                  const uint32_t *posA, const char *const *idA,
                                  const uint32_t *bcA, int m,
                                  const uint32_t *posB, const char *const *idB,
                                  const uint32_t *bcB, int n, int S,
                                  const float *results, float r2limit,
                                  int posWset2)
{
    qo_sink s = {buf, 0, cap};
    char num[32];
    if (with_header)
        sink_puts(&s, "POS2\tPOS1\tID2\tID1\tfreq[2]\tfreq[1]\tLD\n");
    int cnt = 0;
    for (int i = 0; i < n; i++) {
        if (posWset2 == 0)
            cnt++;
        for (int j = cnt; j < m; j++) {
            float v = results[(size_t)i * m + j];
            if (v >= r2limit && v < 100) {
                snprintf(num, sizeof num, "%u\t%u\t", posB[i], posA[j]);
                sink_puts(&s, num);
                sink_puts(&s, idB[i]);
                sink_putc(&s, '\t');
                sink_puts(&s, idA[j]);
                sink_putc(&s, '\t');
                fmt_f(&s, 1.0f * (float)bcB[i] / (float)S, 9);
                sink_putc(&s, '\t');
                fmt_f(&s, 1.0f * (float)bcA[j] / (float)S, 9);
                sink_putc(&s, '\t');
                fmt_f(&s, v, 9);
                sink_putc(&s, '\n');
            }
        }
    }
    return s.len;
}

/* ----------------------------------------------------------- COUNTSTATES -- */

/*
 * countStates_mode (correlate_IO.c:472-516), pair (A row a, B row b): st
 * starts at 0; for every word k, bit p = 0..63 ORs 1 << (bitA*2 + bitB) into
 * st (stopping early once st == 15), and st is then replaced by its own
 * popcount -- so the next word starts from that count read as a bit set.
 * Written as the reference's loop; out[b*m + a] (B-major like r^2).
 */
QO_EXPORT void qo_count_states(const uint64_t *A, int m, const uint64_t *B, int n, int K,
                               uint8_t *out)
{
#pragma omp parallel for schedule(dynamic, 4)
    for (int b = 0; b < n; b++) {
        for (int a = 0; a < m; a++) {
            uint8_t st = 0;
            for (int k = 0; k < K; k++) {
                const uint64_t wa = A[(size_t)a * K + k], wb = B[(size_t)b * K + k];
                for (int p = 0; p < 64; p++) {
                    if (st == 15)
                        break;
                    st |= (uint8_t)(1u << (((wa >> p) & 1u) * 2 + ((wb >> p) & 1u)));
                }
                st = (uint8_t)__builtin_popcount(st);
            }
            out[(size_t)b * m + a] = st;
        }
    }
}

/*
 * writeStateCount (correlate_IO.c:430-470): header, then for B row i and A
 * row j (j > i when posWset2 == 0) "POS2\tPOS1\tID2\tID1\t<states>\t\n".
 * Returns the byte count; writes at most cap bytes.
 */
QO_EXPORT size_t qo_write_states(char *buf, size_t cap, const uint32_t *posA, char **idA, int m,
                                 const uint32_t *posB, char **idB, int n, const uint8_t *st,
                                 int posWset2)
{
    qo_sink s = {buf, 0, cap};
    sink_puts(&s, "POS2\tPOS1\tID2\tID1\tNo_STATES\n");
    char num[16];
    for (int i = 0; i < n; i++) {
        for (int j = posWset2 == 0 ? i + 1 : 0; j < m; j++) {
            snprintf(num, sizeof num, "%u", posB[i]);
            sink_puts(&s, num);
            sink_putc(&s, '\t');
            snprintf(num, sizeof num, "%u", posA[j]);
            sink_puts(&s, num);
            sink_putc(&s, '\t');
            sink_puts(&s, idB[i]);
            sink_putc(&s, '\t');
            sink_puts(&s, idA[j]);
            sink_putc(&s, '\t');
            snprintf(num, sizeof num, "%u", (unsigned)st[(size_t)i * m + j]);
            sink_puts(&s, num);
            sink_puts(&s, "\t\n");
        }
    }
    return s.len;
}

/* ------------------------------------------------------------ VCF -> MDF -- */

/*
 * qLD-parse-2MDF's per-site processing (src/mdf_extension/src/process_data.c:
 * 152-328, snip_processing.c:270-797), restated step by step for the sites a
 * host parser hands over (sample fields of one VCF line, GT position, REF/ALT
 * states).  Random draws use libc rand() as qLD does; seed with qo_srand.
 * Returns 0, or the index of the first site qLD would stop on (with *what
 * set to a short reason).
 */
typedef struct qo_site {
    long long off;
    int len, gt_pos, n_states;
    char states[4];
} qo_site;

QO_EXPORT void qo_srand(unsigned seed) { srand(seed); }

/* getGTfield: keep subfield `pos` in place; returns separators + 1. */
static int qo_gt_field(char *s, int pos)
{
    int len = (int)strlen(s), j = 0, counter = 0;
    for (int i = 0; i < len; i++) {
        if (s[i] != ':') {
            if (pos == 0) {
                s[j++] = s[i];
                if (s[i] == '|' || s[i] == '/')
                    counter++;
            }
        } else {
            pos--;
            if (pos == -1) {
                s[j] = 0;
                break;
            }
        }
    }
    return counter + 1;
}

static void qo_shuffle(char *d, int start, int end)
{
    if (start == end)
        return;
    for (int i = end; i > start; i--) {
        int idx = start + (rand() % (i - start + 1));
        char t = d[idx];
        d[idx] = d[i];
        d[i] = t;
    }
}

/* getGTdata; returns 0 or an error reason. */
static const char *qo_gt_data(const char *s, const char *states, int nstates, char *out)
{
    int len = (int)strlen(s), j = 0, start = 0, end = 0;
    for (int i = 0; i < len; i++) {
        if (s[i] >= '0' && s[i] <= '9') {
            if (s[i] - '0' >= nstates)
                return "allele index past the REF/ALT states";
            if (j + 1 >= 4)
                return "more than three alleles in a genotype";
            out[j++] = states[s[i] - '0'];
        } else {
            if (s[i] == '.') {
                if (j + 1 >= 4)
                    return "more than three alleles in a genotype";
                out[j++] = 'N';
            }
            if (s[i] == '/')
                end++;
            if (s[i] == '|') {
                qo_shuffle(out, start, end);
                start = j;
                end = j;
            }
        }
    }
    qo_shuffle(out, start, end);
    out[j] = 0;
    return 0;
}

static int qo_map(char a)
{
    switch (a) {
    case '0': return 0;
    case '1': return 1;
    case '-': case 'N': return 2;
    case 'A': return 3;
    case 'C': return 4;
    case 'G': return 5;
    case 'T': return 6;
    default: return -1;
    }
}

QO_EXPORT int qo_vcf_pack(const char *text, const qo_site *sites, int nsites,
                          const uint8_t *valid, int nsamples, int ploidy, int K,
                          uint64_t *words, uint32_t *bc, int *snip_len, uint8_t *keep,
                          const char **what)
{
    static char reason[128];
    *what = "";
    size_t cap = (size_t)nsamples * 4 + 16;
    char *snip = malloc(cap), *word = malloc(1 << 16);
    int fail = -1;
    for (int s = 0; s < nsites && fail < 0; s++) {
        const qo_site *st = &sites[s];
        char states[5] = {'X', 'X', 'X', 'X', 'X'};
        for (int k = 0; k < st->n_states && k < 4; k++)
            states[k] = st->states[k];
        snip[0] = 0;
        size_t sl = 0;
        int sample = 0;
        const char *t = text + st->off;
        int i = 0;
        /* getWordFromString over the segment: runs of spaces/tabs separate */
        while (i < st->len) {
            while (i < st->len && (t[i] == ' ' || t[i] == '\t'))
                i++;
            if (i >= st->len)
                break;
            int w = 0;
            while (i < st->len && t[i] != ' ' && t[i] != '\t' && w < (1 << 16) - 1)
                word[w++] = t[i++];
            word[w] = 0;
            if (sample >= nsamples) {
                *what = "more sample fields than header samples";
                fail = s;
                break;
            }
            if (valid[sample]) {
                const int size = qo_gt_field(word, st->gt_pos);
                if (word[0] == 0) {
                    *what = "empty GT field";
                    fail = s;
                    break;
                }
                if (size > ploidy) {
                    *what = "Detected data bigger than the ploidy of input";
                    fail = s;
                    break;
                }
                char part[8];
                const char *e = qo_gt_data(word, states, st->n_states, part);
                if (e) {
                    *what = e;
                    fail = s;
                    break;
                }
                if ((int)strlen(part) < size) {
                    *what = "a genotype with fewer alleles than separators";
                    fail = s;
                    break;
                }
                memcpy(snip + sl, part, (size_t)size);
                sl += (size_t)size;
                snip[sl] = 0;
            }
            sample++;
        }
        if (fail >= 0)
            break;
        const int L = (int)sl;
        snip_len[s] = L;
        keep[s] = 0;
        bc[s] = 0;
        memset(words + (size_t)s * K, 0, sizeof(uint64_t) * (size_t)K);
        if (L == 0) {
            *what = "no alleles (empty alignment)";
            fail = s;
            break;
        }
        if (L > K * 64) {
            *what = "Detected data bigger than the ploidy of input";
            fail = s;
            break;
        }
        /* determineStates / getDataType */
        int cnt[8] = {0};
        for (int q = 0; q < L; q++) {
            const int m = qo_map(snip[q]);
            if (m < 0) {
                snprintf(reason, sizeof reason, "a state character qLD cannot map (%c)", snip[q]);
                *what = reason;
                fail = s;
                break;
            }
            cnt[m]++;
        }
        if (fail >= 0)
            break;
        int acgt = cnt[3] + cnt[4] + cnt[5] + cnt[6], type;
        if ((cnt[0] || cnt[1]) && acgt == 0)
            type = cnt[2] ? 3 : 2;
        else if (acgt && cnt[0] + cnt[1] == 0)
            type = cnt[2] ? 5 : 4;
        else if (cnt[2])
            type = 6;
        else
            type = 0;
        /* removeNonPolymorphicSite with filterOut = 0 */
        int rm = 0;
        if (type == 4 || type == 5 || type == 2 || type == 3) {
            int setv[8] = {0};
            rm = 1;
            const int dna = type >= 4;
            for (int q = 0; q < L; q++) {
                setv[qo_map(snip[q])]++;
                const int dif = dna ? (setv[3] != 0) + (setv[4] != 0) + (setv[5] != 0) +
                                          (setv[6] != 0)
                                    : (setv[0] != 0) + (setv[1] != 0);
                if (dif >= 2) {
                    rm = 0;
                    break;
                }
            }
            if (setv[2])
                rm = 1;
        } else if (type == 6) {
            rm = 1;
        }
        if (rm)
            continue;
        /* binaryDeduction: two bases here, so minorToMajor changes nothing;
         * convertAlignmentBIN: the first base -> '0', the other -> '1' */
        if (type == 4 || type == 5) {
            char s0 = 'x', s1 = 'x';
            int distinct = 0;
            int seen[8] = {0};
            for (int q = 0; q < L; q++) {
                const int m = qo_map(snip[q]);
                if (m >= 3 && !seen[m]) {
                    seen[m] = 1;
                    distinct++;
                }
            }
            if (distinct > 2) {
                *what = "more than two bases at a site";
                fail = s;
                break;
            }
            if (distinct == 2)
                for (int q = 0; q < L; q++) {
                    const char c = snip[q];
                    if (s0 == 'x' && c != '-' && c != 'N')
                        s0 = c;
                    if (s0 != 'x' && s1 == 'x' && c != s0 && c != '-' && c != 'N')
                        s1 = c;
                    snip[q] = c == '-' ? '-' : c == 'N' ? 'N' : c == s0 ? '0' : c == s1 ? '1' : 'X';
                }
        }
        /* compressSnip_x64: bit = character & 1, MSB first */
        uint64_t *w = words + (size_t)s * K, tmp = 0;
        int nb = 0, wi = 0;
        uint32_t ones = 0;
        for (int q = 0; q < L; q++) {
            const uint64_t b = (uint64_t)((unsigned char)snip[q] & 1u);
            tmp = (tmp << 1) | b;
            ones += (uint32_t)b;
            if (++nb == 64) {
                w[wi++] = tmp;
                tmp = 0;
                nb = 0;
            }
        }
        if (nb)
            w[wi] = tmp << (64 - nb);
        bc[s] = ones;
        keep[s] = 1;
    }
    free(snip);
    free(word);
    return fail;
}
