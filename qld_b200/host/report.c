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
 * the blocks are written in order.  Rows come from a dense r^2 array
 * (qld_report_write) or from qld_cuda_ld_hits blocks, whose mask bits and
 * packed values are already filtered on the GPU (qld_report_hits).
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

/* One report line: POS2 POS1 ID2 ID1 freq[2] freq[1] LD. */
static int emit(block *b, const rowtxt *bt, const rowtxt *at, float v)
{
    if (ensure(b, (size_t)bt->pos_n + at->pos_n + bt->id_n + at->id_n + bt->freq_n +
                      at->freq_n + 64))
        return -1;
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
    return 0;
}

/* Rows [row0, row0 + n) of B, from a dense r^2 block (r2 row i at
 * r2 + i*m, kept if r2limit <= v < 100 and, with `single`, j > row0 + i) or
 * from a qld_cuda_ld_hits block (mask bits and packed values). */
typedef struct rep_job {
    const uint8_t *states;     /* COUNTSTATES rows instead of r^2 */
    const float *r2;
    float r2limit;
    int single;
    const qld_hits_block *hits;
    int m, n, row0;
    const rowtxt *ta, *tb;     /* tb indexed by B row */
    block *blocks;
    int nblocks, rows_per_block;
    atomic_int next;
    atomic_int failed;
} rep_job;

/* writeStateCount's line: POS2 POS1 ID2 ID1 <states> and a trailing tab. */
static int emit_states(block *b, const rowtxt *bt, const rowtxt *at, unsigned st)
{
    if (ensure(b, (size_t)bt->pos_n + at->pos_n + bt->id_n + at->id_n + 16))
        return -1;
    char *o = b->buf + b->len;
    memcpy(o, bt->pos, bt->pos_n); o += bt->pos_n; *o++ = '\t';
    memcpy(o, at->pos, at->pos_n); o += at->pos_n; *o++ = '\t';
    memcpy(o, bt->id, bt->id_n); o += bt->id_n; *o++ = '\t';
    memcpy(o, at->id, at->id_n); o += at->id_n; *o++ = '\t';
    char d[4];
    int nd = 0;
    do {
        d[nd++] = (char)('0' + st % 10);
        st /= 10;
    } while (st);
    while (nd)
        *o++ = d[--nd];
    *o++ = '\t';
    *o++ = '\n';
    b->len = (size_t)(o - b->buf);
    return 0;
}

static int format_row(const rep_job *j, int i, block *b)
{
    const int gi = j->row0 + i;
    const rowtxt *bt = &j->tb[gi];
    if (j->states) {
        const uint8_t *row = j->states + (size_t)i * j->m;
        for (int c = j->single ? gi + 1 : 0; c < j->m; ++c)
            if (emit_states(b, bt, &j->ta[c], row[c]))
                return -1;
        return 0;
    }
    if (j->hits) {
        const qld_hits_block *h = j->hits;
        const uint32_t *mw = h->mask + (size_t)i * h->words;
        const float *v = h->val + h->row_off[i];
        for (int w = 0; w < h->words; ++w)
            for (uint32_t bits = mw[w]; bits; bits &= bits - 1) {
                const int c = w * 32 + __builtin_ctz(bits);
                if (emit(b, bt, &j->ta[c], *v++))
                    return -1;
            }
        return 0;
    }
    const float *row = j->r2 + (size_t)i * j->m;
    for (int c = j->single ? gi + 1 : 0; c < j->m; ++c) {
        const float v = row[c];
        if (v >= j->r2limit && v < 100 && emit(b, bt, &j->ta[c], v))
            return -1;
    }
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
        for (int i = i0; i < i1; ++i)
            if (format_row(j, i, b)) {
                atomic_store(&j->failed, 1);
                return NULL;
            }
    }
    return NULL;
}

struct qld_report {
    FILE *fp;
    const qld_table *A, *B;
    rowtxt *ta, *tb;
    char *pa, *pb;
    int snip_size, threads, per_round, rows_per_block;
    block *blocks;
};

int qld_report_open(qld_report **out, FILE *fp, const qld_table *A, const qld_table *B,
                    int snip_size, int threads)
{
    if (!out)
        return qld_host_fail(QLD_ERR_INVALID, "NULL report handle");
    *out = NULL;
    if (!fp || !A || !B || snip_size < 1)
        return qld_host_fail(QLD_ERR_INVALID, "bad report arguments");
    qld_report *r = calloc(1, sizeof *r);
    if (!r)
        return qld_host_fail(QLD_ERR_NOMEM, "out of memory");
    r->fp = fp;
    r->A = A;
    r->B = B;
    r->snip_size = snip_size;
    r->threads = threads < 1 ? 1 : threads;
    r->rows_per_block = 64;
    r->per_round = r->threads * 4;   /* row blocks formatted before each write-out */
    r->blocks = calloc((size_t)r->per_round, sizeof *r->blocks);
    if (!r->blocks || row_texts(A, snip_size, &r->ta, &r->pa) ||
        (B == A ? (r->tb = r->ta, 0) : row_texts(B, snip_size, &r->tb, &r->pb))) {
        qld_report_close(r);
        return qld_host_fail(QLD_ERR_NOMEM, "out of memory");
    }
    if (fputs("POS2\tPOS1\tID2\tID1\tfreq[2]\tfreq[1]\tLD\n", fp) == EOF) {
        qld_report_close(r);
        return qld_host_fail(QLD_ERR_INVALID, "write failed");
    }
    *out = r;
    return QLD_OK;
}

/* Format rows [row0, row0 + n) with the report's threads and write them in
 * order, per_round row blocks at a time. */
static int run_rows(qld_report *r, rep_job *proto, int row0, int n)
{
    const int span = r->rows_per_block * r->per_round;
    for (int i0 = 0; i0 < n; i0 += span) {
        const int rows = n - i0 < span ? n - i0 : span;
        rep_job j = *proto;
        j.row0 = row0 + i0;
        j.n = rows;
        if (j.r2)
            j.r2 = proto->r2 + (size_t)i0 * j.m;
        if (j.states)
            j.states = proto->states + (size_t)i0 * j.m;
        qld_hits_block sub;
        if (proto->hits) {   /* the same block seen from local row i0 */
            sub = *proto->hits;
            sub.mask += (size_t)i0 * sub.words;
            sub.row_off += i0;
            j.hits = &sub;
        }
        j.ta = r->ta;
        j.tb = r->tb;
        j.blocks = r->blocks;
        j.rows_per_block = r->rows_per_block;
        j.nblocks = (rows + r->rows_per_block - 1) / r->rows_per_block;
        atomic_init(&j.next, 0);
        atomic_init(&j.failed, 0);
        for (int k = 0; k < j.nblocks; ++k)
            r->blocks[k].len = 0;
        qld_run_threads(rep_worker, &j, r->threads < j.nblocks ? r->threads : j.nblocks);
        if (atomic_load(&j.failed))
            return qld_host_fail(QLD_ERR_NOMEM, "out of memory");
        for (int k = 0; k < j.nblocks; ++k)
            if (r->blocks[k].len &&
                fwrite(r->blocks[k].buf, 1, r->blocks[k].len, r->fp) != r->blocks[k].len)
                return qld_host_fail(QLD_ERR_INVALID, "write failed");
    }
    return QLD_OK;
}

int qld_report_hits(qld_report *r, const qld_hits_block *blk)
{
    if (!r || !blk || blk->rows < 0 || blk->row0 < 0 || blk->row0 + blk->rows > r->B->rows ||
        blk->m != r->A->rows || (blk->rows && (!blk->mask || !blk->row_off)))
        return qld_host_fail(QLD_ERR_INVALID, "block does not match the report's tables");
    rep_job proto;
    memset(&proto, 0, sizeof proto);
    proto.hits = blk;
    proto.m = blk->m;
    return run_rows(r, &proto, blk->row0, blk->rows);
}

int qld_report_close(qld_report *r)
{
    if (!r)
        return QLD_OK;
    for (int k = 0; r->blocks && k < r->per_round; ++k)
        free(r->blocks[k].buf);
    free(r->blocks);
    if (r->tb != r->ta) {
        free(r->tb);
        free(r->pb);
    }
    free(r->ta);
    free(r->pa);
    free(r);
    return QLD_OK;
}

int qld_report_write(FILE *fp, const qld_table *A, const qld_table *B, const float *r2,
                     int snip_size, float r2limit, int single_region, int threads)
{
    if (!fp || !A || !B || (!r2 && A->rows && B->rows) || snip_size < 1)
        return qld_host_fail(QLD_ERR_INVALID, "bad report arguments");
    qld_report *r;
    int rc = qld_report_open(&r, fp, A, B, snip_size, threads);
    if (rc != QLD_OK)
        return rc;
    if (A->rows && B->rows) {
        rep_job proto;
        memset(&proto, 0, sizeof proto);
        proto.r2 = r2;
        proto.r2limit = r2limit;
        proto.single = single_region;
        proto.m = A->rows;
        rc = run_rows(r, &proto, 0, B->rows);
    }
    qld_report_close(r);
    return rc;
}

int qld_report_states(FILE *fp, const qld_table *A, const qld_table *B, const uint8_t *states,
                      int single_region, int threads)
{
    if (!fp || !A || !B || (!states && A->rows && B->rows))
        return qld_host_fail(QLD_ERR_INVALID, "bad report arguments");
    qld_report *r = calloc(1, sizeof *r);
    if (!r)
        return qld_host_fail(QLD_ERR_NOMEM, "out of memory");
    r->fp = fp;
    r->A = A;
    r->B = B;
    r->snip_size = 1;
    r->threads = threads < 1 ? 1 : threads;
    r->rows_per_block = 64;
    r->per_round = r->threads * 4;
    r->blocks = calloc((size_t)r->per_round, sizeof *r->blocks);
    int rc = QLD_OK;
    if (!r->blocks || row_texts(A, 1, &r->ta, &r->pa) ||
        (B == A ? (r->tb = r->ta, 0) : row_texts(B, 1, &r->tb, &r->pb)))
        rc = qld_host_fail(QLD_ERR_NOMEM, "out of memory");
    else if (fputs("POS2\tPOS1\tID2\tID1\tNo_STATES\n", fp) == EOF)
        rc = qld_host_fail(QLD_ERR_INVALID, "write failed");
    else if (A->rows && B->rows) {
        rep_job proto;
        memset(&proto, 0, sizeof proto);
        proto.states = states;
        proto.single = single_region;
        proto.m = A->rows;
        rc = run_rows(r, &proto, 0, B->rows);
    }
    qld_report_close(r);
    return rc;
}
