/*
 * mdf_loader.c -- qLD MDF datasets into pinned host memory (qld_host.h).
 *
 * Same selection as qLD-compute's MDF path -- header (readHeaderFile,
 * src/correlator/src/correlate_IO.c:79-259), the parts covering the position
 * window (findFiles, :294-376) and rows with posWmin <= POS <= posWmax read in
 * file order with their BC field and the first K words (readTable_x64 /
 * writeMDF_x64, correlate_IOx64.c:27-122,351-461) -- but parts are parsed in
 * parallel by worker threads with a hand-written decimal parser instead of
 * strtoul and malformed input returns a status instead of exiting.  Words
 * past K on a line are read and ignored: qLD-parse-2MDF pads haploid data to
 * its diploid default width with words it never initialises, and qLD-compute
 * copies them past the row, where the next row overwrites them.
 */
#define _GNU_SOURCE
#include <dirent.h>
#include <errno.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <zlib.h>

#include "host_internal.h"
#include "qld_host.h"

static __thread char g_err[512];

const char *qld_host_last_error(void) { return g_err; }

int qld_host_fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

/* ------------------------------------------------------------------ header -- */

static char *gz_line(gzFile f, char **buf, size_t *cap)
{
    size_t len = 0;
    if (!*buf) {
        *cap = 1 << 16;
        *buf = malloc(*cap);
        if (!*buf)
            return NULL;
    }
    for (;;) {
        if (!gzgets(f, *buf + len, (int)(*cap - len)))
            return len ? *buf : NULL;
        len += strlen(*buf + len);
        if (len && (*buf)[len - 1] == '\n') {
            (*buf)[len - 1] = '\0';
            return *buf;
        }
        if (len + 1 < *cap) /* EOF without newline */
            return *buf;
        char *nb = realloc(*buf, *cap * 2);
        if (!nb)
            return NULL;
        *buf = nb;
        *cap *= 2;
    }
}

static int dir_path(const char *dir, const char *name, char *out, size_t cap)
{
    size_t n = strlen(dir);
    return snprintf(out, cap, "%s%s%s", dir, (n && dir[n - 1] == '/') ? "" : "/", name) <
           (int)cap;
}

/* The dataset's header file: the lexically first regular file whose name
 * contains "header" (qLD's readHeaderFile() takes the one readdir() finds). */
static int header_file(const char *dir, char *name, size_t name_cap, char *path,
                       size_t path_cap)
{
    DIR *dp = opendir(dir);
    if (!dp)
        return qld_host_fail(QLD_ERR_INVALID, "cannot open directory %s", dir);
    name[0] = '\0';
    struct dirent *e;
    while ((e = readdir(dp))) {
        char p[4096];
        struct stat st;
        if (!strstr(e->d_name, "header") || !dir_path(dir, e->d_name, p, sizeof p) ||
            stat(p, &st) || !S_ISREG(st.st_mode))
            continue;
        if (!name[0] || strcmp(e->d_name, name) < 0)
            snprintf(name, name_cap, "%s", e->d_name);
    }
    closedir(dp);
    if (!name[0])
        return qld_host_fail(QLD_ERR_INVALID, "no header file in %s", dir);
    dir_path(dir, name, path, path_cap);
    return QLD_OK;
}

static const char *const kVcfFields[9] = {"#CHROM", "POS", "ID", "REF", "ALT",
                                          "QUAL", "FILTER", "INFO", "FORMAT"};

int qld_mdf_read_header(const char *dir, qld_mdf_header *h)
{
    if (!dir || !h)
        return qld_host_fail(QLD_ERR_INVALID, "NULL argument");
    memset(h, 0, sizeof *h);
    char best[1024], path[4096];
    int rc = header_file(dir, best, sizeof best, path, sizeof path);
    if (rc)
        return rc;
    /* alignment id: the name up to the first '_' (or quote), as sscanf("%[^'_']") */
    size_t k = strcspn(best, "_'");
    if (k == 0 || k >= sizeof h->id)
        return qld_host_fail(QLD_ERR_INVALID, "bad header file name %s", best);
    memcpy(h->id, best, k);
    h->id[k] = '\0';
    gzFile f = gzopen(path, "r");
    if (!f)
        return qld_host_fail(QLD_ERR_INVALID, "cannot open %s", path);
    char *buf = NULL;
    size_t cap = 0;
    rc = qld_host_fail(QLD_ERR_INVALID, "%s: no #CHROM line", path);
    if (!gz_line(f, &buf, &cap)) {
        rc = qld_host_fail(QLD_ERR_INVALID, "%s: empty header", path);
        goto out;
    }
    while (gz_line(f, &buf, &cap)) {
        if (strncmp(buf, "#CHROM", 6) != 0)
            continue;
        int nf = 0;
        for (char *save = NULL, *t = strtok_r(buf, " \t", &save); t;
             t = strtok_r(NULL, " \t", &save), ++nf)
            if (nf < 9 && strcmp(t, kVcfFields[nf]) != 0) {
                rc = qld_host_fail(QLD_ERR_INVALID, "%s: VCF header field %s missing", path,
                                   kVcfFields[nf]);
                goto out;
            }
        h->samples = nf - 9;
        if (h->samples <= 0 || !gz_line(f, &buf, &cap)) {
            rc = qld_host_fail(QLD_ERR_INVALID, "%s: wrong header format", path);
            goto out;
        }
        char id2[256];
        if (sscanf(buf, "%255s %d %d %d %d %d", id2, &h->snips_per_file, &h->snip_size,
                   &h->total_snips, &h->pos_min, &h->pos_max) != 6 ||
            strcmp(id2, h->id) != 0) {
            rc = qld_host_fail(QLD_ERR_INVALID, "%s: bad info line", path);
            goto out;
        }
        rc = QLD_OK;
        break;
    }
out:
    free(buf);
    gzclose(f);
    return rc;
}

int qld_mdf_listed_samples(const char *dir, const char *const *names, int nnames, int *listed)
{
    if (!dir || !listed || nnames < 0 || (nnames > 0 && !names))
        return qld_host_fail(QLD_ERR_INVALID, "bad argument");
    *listed = 0;
    char best[1024], path[4096];
    int rc = header_file(dir, best, sizeof best, path, sizeof path);
    if (rc)
        return rc;
    gzFile f = gzopen(path, "r");
    if (!f)
        return qld_host_fail(QLD_ERR_INVALID, "cannot open %s", path);
    char *buf = NULL;
    size_t cap = 0;
    rc = qld_host_fail(QLD_ERR_INVALID, "%s: no #CHROM line", path);
    while (gz_line(f, &buf, &cap)) {
        if (strncmp(buf, "#CHROM", 6) != 0)
            continue;
        /* makeValidList(): the words after the nine fixed VCF fields; a name
         * counts if it equals an entry of the list (sample_isValid()) */
        int nf = 0, count = 0;
        for (char *save = NULL, *t = strtok_r(buf, " \t\r\n", &save); t;
             t = strtok_r(NULL, " \t\r\n", &save), ++nf) {
            if (nf < 9)
                continue;
            int hit = nnames == 0;
            for (int i = 0; i < nnames && !hit; ++i)
                hit = strcmp(names[i], t) == 0;
            count += hit;
        }
        *listed = count;
        rc = QLD_OK;
        break;
    }
    free(buf);
    gzclose(f);
    return rc;
}

/* ------------------------------------------------------------------- parts -- */

typedef struct part {
    char path[4096];
    int i0, i1, p0, p1;
    /* parse result */
    int rows;
    uint64_t *words;
    uint32_t *bc, *pos;
    char *ids;          /* NUL-separated */
    size_t ids_len;
    int rc;
    char err[512];
    size_t row_off, id_off;
} part;

static int part_cmp(const void *a, const void *b)
{
    return ((const part *)a)->i0 - ((const part *)b)->i0;
}

/* atoi(): optional blanks and sign, then digits. */
static int parse_int(const char *s, const char *e)
{
    while (s < e && (*s == ' ' || *s == '\t'))
        ++s;
    int neg = 0;
    if (s < e && (*s == '-' || *s == '+'))
        neg = *s++ == '-';
    long v = 0;
    while (s < e && *s >= '0' && *s <= '9')
        v = v * 10 + (*s++ - '0');
    return (int)(neg ? -v : v);
}

static int parse_u64(const char *s, const char *e, uint64_t *out)
{
    if (s == e)
        return -1;
    uint64_t v = 0;
    for (; s < e; ++s) {
        if (*s < '0' || *s > '9')
            return -1;
        const uint64_t d = (uint64_t)(*s - '0');
        if (v > (UINT64_MAX - d) / 10)
            return -1;
        v = v * 10 + d;
    }
    *out = v;
    return 0;
}

typedef struct load_job {
    part *parts;
    int nparts;
    int K, pos_min, pos_max;
    atomic_int next;
} load_job;

static int part_fail(part *p, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(p->err, sizeof p->err, fmt, ap);
    va_end(ap);
    p->rc = QLD_ERR_INVALID;
    return p->rc;
}

static int parse_part(part *p, int K, int pos_min, int pos_max)
{
    FILE *f = fopen(p->path, "rb");
    if (!f)
        return part_fail(p, "cannot open %s", p->path);
    fseek(f, 0, SEEK_END);
    long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *text = malloc((size_t)size + 1);
    if (!text || fread(text, 1, (size_t)size, f) != (size_t)size) {
        fclose(f);
        free(text);
        return part_fail(p, "cannot read %s", p->path);
    }
    fclose(f);
    text[size] = '\0';
    size_t lines = 1;
    for (long i = 0; i < size; ++i)
        lines += text[i] == '\n';
    p->words = malloc(sizeof(uint64_t) * (size_t)K * lines);
    p->bc = malloc(sizeof(uint32_t) * lines);
    p->pos = malloc(sizeof(uint32_t) * lines);
    p->ids = malloc((size_t)size + 1);
    if (!p->words || !p->bc || !p->pos || !p->ids) {
        free(text);
        return part_fail(p, "out of memory reading %s", p->path);
    }
    p->rows = 0;
    p->ids_len = 0;
    const char *s = text, *end = text + size;
    for (int ln = 0; s < end; ++ln) {
        const char *e = memchr(s, '\n', (size_t)(end - s));
        if (!e)
            e = end;
        const char *le = e;
        if (le > s && le[-1] == '\r')
            --le;
        /* the first two lines are the MDF header (readTable_x64 skips them); a
         * line parses as CHROM POS ID BC w0 ..., and rows outside the window
         * are skipped.  The '#CHROM' column-name line is skipped as well (qLD
         * reads it as a row at POS 0, which no clamped window contains). */
        if (ln >= 2 && le - s >= 3 && *s != '#') {
            const char *f0 = s, *fe[4];
            const char *fs[4];
            const char *c = f0;
            int nf = 0;
            while (nf < 4) {
                while (c < le && (*c == ' ' || *c == '\t'))
                    ++c;
                if (c >= le)
                    break;
                fs[nf] = c;
                while (c < le && *c != ' ' && *c != '\t')
                    ++c;
                fe[nf++] = c;
            }
            if (nf >= 2) {
                const int pos = parse_int(fs[1], fe[1]);
                if (pos >= pos_min && pos <= pos_max) {
                    if (nf < 4) {
                        free(text);
                        return part_fail(p, "%s line %d: missing ID/BC fields", p->path, ln + 1);
                    }
                    uint64_t *w = p->words + (size_t)p->rows * K;
                    int k = 0;
                    while (c < le) {
                        while (c < le && (*c == ' ' || *c == '\t'))
                            ++c;
                        if (c >= le)
                            break;
                        const char *ws = c;
                        while (c < le && *c != ' ' && *c != '\t')
                            ++c;
                        uint64_t v;
                        if (parse_u64(ws, c, &v)) {
                            free(text);
                            return part_fail(p, "%s line %d: bad word", p->path, ln + 1);
                        }
                        if (k < K)
                            w[k] = v;
                        ++k;
                    }
                    if (k < K) {
                        free(text);
                        return part_fail(p, "%s line %d: %d words, %d needed", p->path, ln + 1,
                                         k, K);
                    }
                    p->pos[p->rows] = (uint32_t)pos;
                    p->bc[p->rows] = (uint32_t)parse_int(fs[3], fe[3]);
                    memcpy(p->ids + p->ids_len, fs[2], (size_t)(fe[2] - fs[2]));
                    p->ids_len += (size_t)(fe[2] - fs[2]);
                    p->ids[p->ids_len++] = '\0';
                    ++p->rows;
                }
            }
        }
        s = e + 1;
    }
    free(text);
    p->rc = QLD_OK;
    return QLD_OK;
}

static void *load_worker(void *arg)
{
    load_job *j = arg;
    for (;;) {
        int i = atomic_fetch_add(&j->next, 1);
        if (i >= j->nparts)
            break;
        parse_part(&j->parts[i], j->K, j->pos_min, j->pos_max);
    }
    return NULL;
}

typedef struct copy_job {
    part *parts;
    int nparts, K;
    qld_table *t;
    atomic_int next;
} copy_job;

static void *copy_worker(void *arg)
{
    copy_job *j = arg;
    for (;;) {
        int i = atomic_fetch_add(&j->next, 1);
        if (i >= j->nparts)
            break;
        part *p = &j->parts[i];
        memcpy(j->t->words + p->row_off * j->K, p->words, sizeof(uint64_t) * j->K * p->rows);
        memcpy(j->t->bc + p->row_off, p->bc, sizeof(uint32_t) * p->rows);
        memcpy(j->t->pos + p->row_off, p->pos, sizeof(uint32_t) * p->rows);
        memcpy(j->t->id_pool + p->id_off, p->ids, p->ids_len);
        char *q = j->t->id_pool + p->id_off;
        for (int r = 0; r < p->rows; ++r) {
            j->t->ids[p->row_off + r] = q;
            q += strlen(q) + 1;
        }
    }
    return NULL;
}

void qld_run_threads(void *(*fn)(void *), void *arg, int threads)
{
    if (threads < 1)
        threads = 1;
    pthread_t *tid = calloc((size_t)threads, sizeof *tid);
    int created = 0;
    for (int i = 0; tid && i < threads - 1; ++i)
        if (pthread_create(&tid[created], NULL, fn, arg) == 0)
            ++created;
    fn(arg);
    for (int i = 0; i < created; ++i)
        pthread_join(tid[i], NULL);
    free(tid);
}

int qld_mdf_load(qld_ctx *ctx, const char *dir, int pos_min, int pos_max, int K, int threads,
                 qld_table *out)
{
    if (!dir || !out || K < 1)
        return qld_host_fail(QLD_ERR_INVALID, "bad arguments");
    memset(out, 0, sizeof *out);
    qld_mdf_header h;
    int rc = qld_mdf_read_header(dir, &h);
    if (rc)
        return rc;
    DIR *dp = opendir(dir);
    if (!dp)
        return qld_host_fail(QLD_ERR_INVALID, "cannot open directory %s", dir);
    int cap = 64, np = 0;
    part *parts = calloc((size_t)cap, sizeof *parts);
    struct dirent *e;
    while (parts && (e = readdir(dp))) {
        char id[256];
        int i0, i1, p0, p1;
        if (!strstr(e->d_name, h.id) || strstr(e->d_name, "header") || !strstr(e->d_name, ".mdf"))
            continue;
        if (sscanf(e->d_name, "%255[^_]_%d_%d_%d_%d.", id, &i0, &i1, &p0, &p1) != 5 ||
            strcmp(id, h.id) != 0)
            continue;
        if (p1 < pos_min || p0 > pos_max)
            continue;
        if (np == cap) {
            part *nb = realloc(parts, sizeof *parts * (size_t)cap * 2);
            if (!nb)
                break;
            memset(nb + cap, 0, sizeof *parts * (size_t)cap);
            parts = nb;
            cap *= 2;
        }
        part *p = &parts[np++];
        p->i0 = i0; p->i1 = i1; p->p0 = p0; p->p1 = p1;
        dir_path(dir, e->d_name, p->path, sizeof p->path);
    }
    closedir(dp);
    if (!parts)
        return qld_host_fail(QLD_ERR_NOMEM, "out of memory");
    qsort(parts, (size_t)np, sizeof *parts, part_cmp);
    load_job lj = {parts, np, K, pos_min, pos_max, 0};
    qld_run_threads(load_worker, &lj, threads < np ? threads : (np ? np : 1));
    size_t rows = 0, idb = 0;
    rc = QLD_OK;
    for (int i = 0; i < np; ++i) {
        if (parts[i].rc != QLD_OK && rc == QLD_OK)
            rc = qld_host_fail(parts[i].rc, "%s", parts[i].err);
        parts[i].row_off = rows;
        parts[i].id_off = idb;
        rows += (size_t)parts[i].rows;
        idb += parts[i].ids_len;
    }
    if (rc == QLD_OK && rows > 0x7fffffff)
        rc = qld_host_fail(QLD_ERR_INVALID, "too many rows");
    if (rc == QLD_OK) {
        out->rows = (int)rows;
        out->K = K;
        const size_t wbytes = sizeof(uint64_t) * (size_t)K * (rows ? rows : 1);
        if (ctx) {
            rc = qld_cuda_host_alloc(ctx, wbytes, (void **)&out->words);
            out->pinned = rc == QLD_OK;
        } else if (posix_memalign((void **)&out->words, 64, wbytes)) {
            out->words = NULL;
            rc = QLD_ERR_NOMEM;
        }
        if (rc != QLD_OK) {
            qld_host_fail(rc, "allocation of %zu rows failed", rows);
        } else {
            out->bc = malloc(sizeof(uint32_t) * (rows ? rows : 1));
            out->pos = malloc(sizeof(uint32_t) * (rows ? rows : 1));
            out->ids = malloc(sizeof(char *) * (rows ? rows : 1));
            out->id_pool = malloc(idb ? idb : 1);
            if (!out->bc || !out->pos || !out->ids || !out->id_pool)
                rc = qld_host_fail(QLD_ERR_NOMEM, "out of memory");
        }
        if (rc == QLD_OK) {
            copy_job cj = {parts, np, K, out, 0};
            qld_run_threads(copy_worker, &cj, threads < np ? threads : (np ? np : 1));
        }
    }
    for (int i = 0; i < np; ++i) {
        free(parts[i].words);
        free(parts[i].bc);
        free(parts[i].pos);
        free(parts[i].ids);
    }
    free(parts);
    if (rc != QLD_OK)
        qld_table_free(ctx, out);
    return rc;
}

void qld_table_free(qld_ctx *ctx, qld_table *t)
{
    if (!t)
        return;
    if (t->words && t->pinned)
        qld_cuda_host_free(ctx, t->words);
    else
        free(t->words);
    free(t->bc);
    free(t->pos);
    free(t->ids);
    free(t->id_pool);
    memset(t, 0, sizeof *t);
}
