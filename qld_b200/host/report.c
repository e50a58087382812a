/*
 * report.c -- qLD-compute's text report, multithreaded (qld_host.h).
 *
 * Same bytes as writeResultsHeader()/writeResults() (src/correlator/src/
 * correlate_IO.c:378-429) with fprint_f() (fast_print.c:35-103): rows for B
 * row i (outer) and A row j (inner; j > i for a single region) whose
 * r^2 satisfies r2limit <= r^2 < 100, as
 * POS2 \t POS1 \t ID2 \t ID1 \t freq[2] \t freq[1] \t LD.
 * The per-row pieces (positions, IDs, the two frequencies) are formatted once
 * per row; worker threads format blocks of B rows into private buffers and
 * the blocks are written in order.
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#include "host_internal.h"
#include "qld_host.h"

/* fprint_f semantics: the value times 10^precision is formed in float and
 * truncated (never rounded); the integer part is printed, then '.', then --
 * unless the fraction is zero -- the fraction zero-padded to `precision`
 * digits.  Digits are produced by reversing the decimal digits of the
 * positive parts, so a part <= 0 prints as nothing ("0." for the integer). */
static unsigned rev10(long *v)
{
    unsigned n = 0;
    long r = 0;
    while (*v > 0) {
        ++n;
        r = r * 10 + *v % 10;
        *v /= 10;
    }
    *v = r;
    return n;
}

static size_t fmt_f(char *o, float val, int precision)
{
    size_t k = 0;
    unsigned long p10 = 1;
    for (int j = 0; j < precision; ++j)
        p10 *= 10;
    long scaled = (long)(val * (float)p10);
    long ip = (long)val;
    scaled = (long)((unsigned long)scaled - (unsigned long)ip * p10);
    const unsigned idig = rev10(&ip);
    const unsigned ddig = rev10(&scaled);
    if (ip == 0) {
        o[k++] = '0';
    } else {
        unsigned printed = 0;
        while (ip != 0) {
            o[k++] = (char)('0' + ip % 10);
            ip /= 10;
            ++printed;
        }
        for (unsigned j = 0; j < idig - printed; ++j)
            o[k++] = '0';
    }
    o[k++] = '.';
    if (scaled == 0)
        return k;
    for (unsigned j = 0; j < (unsigned)precision - ddig; ++j)
        o[k++] = '0';
    for (unsigned j = 0; j < ddig; ++j) {
        o[k++] = (char)('0' + scaled % 10);
        scaled /= 10;
    }
    return k;
}

typedef struct rowtxt {
    char *pos, *id, *freq;   /* NUL-terminated */
    unsigned short pos_n, id_n, freq_n;
} rowtxt;

static int row_texts(const qld_table *t, int snip_size, rowtxt **out, char **pool)
{
    size_t bytes = 0;
    for (int r = 0; r < t->rows; ++r)
        bytes += 12 + strlen(t->ids[r]) + 1 + 40;
    rowtxt *rt = malloc(sizeof *rt * (size_t)(t->rows ? t->rows : 1));
    char *p = malloc(bytes ? bytes : 1);
    if (!rt || !p) {
        free(rt);
        free(p);
        return -1;
    }
    char *q = p;
    for (int r = 0; r < t->rows; ++r) {
        rt[r].pos = q;
        rt[r].pos_n = (unsigned short)sprintf(q, "%u", t->pos[r]);
        q += rt[r].pos_n + 1;
        rt[r].id = q;
        size_t n = strlen(t->ids[r]);
        memcpy(q, t->ids[r], n + 1);
        rt[r].id_n = (unsigned short)n;
        q += n + 1;
        rt[r].freq = q;
        rt[r].freq_n = (unsigned short)fmt_f(q, 1.0f * (float)t->bc[r] / (float)snip_size, 9);
        q[rt[r].freq_n] = '\0';
        q += rt[r].freq_n + 1;
    }
    *out = rt;
    *pool = p;
    return 0;
}

typedef struct block {
    char *buf;
    size_t len, cap;
} block;

typedef struct rep_job {
    const float *r2;
    int m, n, row0, single;   /* row0: B row of local row 0 */
    float r2limit;
    const rowtxt *ta, *tb;
    block *blocks;
    int nblocks, rows_per_block;
    atomic_int next;
    atomic_int failed;
} rep_job;

static int ensure(block *b, size_t extra)
{
    if (b->len + extra <= b->cap)
        return 0;
    size_t nc = b->cap ? b->cap : (1 << 20);
    while (nc < b->len + extra)
        nc *= 2;
    char *nb = realloc(b->buf, nc);
    if (!nb)
        return -1;
    b->buf = nb;
    b->cap = nc;
    return 0;
}

static void *rep_worker(void *arg)
{
    rep_job *j = arg;
    for (;;) {
        int bi = atomic_fetch_add(&j->next, 1);
        if (bi >= j->nblocks)
            break;
        block *b = &j->blocks[bi];
        const int i0 = bi * j->rows_per_block;
        const int i1 = i0 + j->rows_per_block < j->n ? i0 + j->rows_per_block : j->n;
        for (int i = i0; i < i1; ++i) {
            const rowtxt *bt = &j->tb[i];
            const float *row = j->r2 + (size_t)i * j->m;
            for (int c = j->single ? j->row0 + i + 1 : 0; c < j->m; ++c) {
                const float v = row[c];
                if (!(v >= j->r2limit && v < 100))
                    continue;
                const rowtxt *at = &j->ta[c];
                if (ensure(b, (size_t)bt->pos_n + at->pos_n + bt->id_n + at->id_n + bt->freq_n +
                                  at->freq_n + 64)) {
                    atomic_store(&j->failed, 1);
                    return NULL;
                }
                char *o = b->buf + b->len;
                memcpy(o, bt->pos, bt->pos_n); o += bt->pos_n; *o++ = '\t';
                memcpy(o, at->pos, at->pos_n); o += at->pos_n; *o++ = '\t';
                memcpy(o, bt->id, bt->id_n); o += bt->id_n; *o++ = '\t';
                memcpy(o, at->id, at->id_n); o += at->id_n; *o++ = '\t';
                memcpy(o, bt->freq, bt->freq_n); o += bt->freq_n; *o++ = '\t';
                memcpy(o, at->freq, at->freq_n); o += at->freq_n; *o++ = '\t';
                o += fmt_f(o, v, 9);
                *o++ = '\n';
                b->len = (size_t)(o - b->buf);
            }
        }
    }
    return NULL;
}

int qld_report_write(FILE *fp, const qld_table *A, const qld_table *B, const float *r2,
                     int snip_size, float r2limit, int single_region, int threads)
{
    if (!fp || !A || !B || (!r2 && A->rows && B->rows) || snip_size < 1)
        return qld_host_fail(QLD_ERR_INVALID, "bad report arguments");
    if (fputs("POS2\tPOS1\tID2\tID1\tfreq[2]\tfreq[1]\tLD\n", fp) == EOF)
        return qld_host_fail(QLD_ERR_INVALID, "write failed");
    if (!A->rows || !B->rows)
        return QLD_OK;
    rowtxt *ta = NULL, *tb = NULL;
    char *pa = NULL, *pb = NULL;
    if (row_texts(A, snip_size, &ta, &pa) ||
        (B == A ? (tb = ta, pb = NULL, 0) : row_texts(B, snip_size, &tb, &pb))) {
        free(ta);
        free(pa);
        return qld_host_fail(QLD_ERR_NOMEM, "out of memory");
    }
    if (threads < 1)
        threads = 1;
    const int rows_per_block = 64;
    const int per_round = threads * 4;   /* blocks formatted before each write-out */
    block *blocks = calloc((size_t)per_round, sizeof *blocks);
    int rc = blocks ? QLD_OK : qld_host_fail(QLD_ERR_NOMEM, "out of memory");
    for (int i0 = 0; rc == QLD_OK && i0 < B->rows; i0 += rows_per_block * per_round) {
        const int rows = B->rows - i0 < rows_per_block * per_round ? B->rows - i0
                                                                   : rows_per_block * per_round;
        rep_job j;
        j.r2 = r2 + (size_t)i0 * A->rows;
        j.m = A->rows;
        j.n = rows;
        j.row0 = i0;
        j.single = single_region;
        j.r2limit = r2limit;
        j.ta = ta;
        j.tb = tb + i0;
        j.blocks = blocks;
        j.rows_per_block = rows_per_block;
        j.nblocks = (rows + rows_per_block - 1) / rows_per_block;
        atomic_init(&j.next, 0);
        atomic_init(&j.failed, 0);
        for (int k = 0; k < j.nblocks; ++k)
            blocks[k].len = 0;
        qld_run_threads(rep_worker, &j, threads < j.nblocks ? threads : j.nblocks);
        if (atomic_load(&j.failed)) {
            rc = qld_host_fail(QLD_ERR_NOMEM, "out of memory");
            break;
        }
        for (int k = 0; k < j.nblocks; ++k)
            if (blocks[k].len && fwrite(blocks[k].buf, 1, blocks[k].len, fp) != blocks[k].len) {
                rc = qld_host_fail(QLD_ERR_INVALID, "write failed");
                break;
            }
    }
    for (int k = 0; blocks && k < per_round; ++k)
        free(blocks[k].buf);
    free(blocks);
    if (tb != ta) {
        free(tb);
        free(pb);
    }
    free(ta);
    free(pa);
    return rc;
}
