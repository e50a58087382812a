/*
 * vcf.c -- the host half of VCF -> MDF conversion (qld_host.h): qLD-parse-
 * VCF's part datasets read and filtered line by line, the MDF parts written.
 *
 * Follows qLD-parse-2MDF (src/mdf_extension/src):
 *   header       readHeaderFile (io.c:148-333): the first "*header*" file,
 *                alignment id = its name up to '_' or '\'', line 1, the
 *                #CHROM line with the nine fixed names and the sample names
 *                (valid mask from the sample list, valid count += ploidy per
 *                valid sample), then "<id> snipsPerFile snipSize totalSnips";
 *   parts        findFiles + sort_files (io.c:19-52,337-374): names holding
 *                the id, ".vcf.gz" and no "header", prefix before '_' equal
 *                to the id, ordered by the first number after '_';
 *   lines        readTable_x64 + writeToTable_x64's fixed fields
 *                (process_data.c:27-150,329-393): the two header lines must
 *                match, lines shorter than 3 characters are ignored, words
 *                split on runs of spaces and tabs (read_file.c:53-137), and a
 *                line is skipped for a multi-character or symbolic REF/ALT, a
 *                FILTER other than PASS or '.', an INFO AF of exactly 0 or 1 or
 *                a VT other than SNP, or a FORMAT without GT
 *                (snip_processing.c:43-304);
 *   output       the MDF text of process_data.c:441-460.
 * Input the reference rejects with assert/exit is a QLD_ERR_INVALID status
 * with a message here.  The sample fields are left to the GPU
 * (qld_cuda_vcf_pack).
 */
#define _GNU_SOURCE
#include <dirent.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <zlib.h>

#include "host_internal.h"
#include "qld_host.h"

static const char *const kFixed[9] = {"#CHROM", "POS",    "ID",   "REF",   "ALT",
                                      "QUAL",   "FILTER", "INFO", "FORMAT"};

static int is_sep(char c) { return c == ' ' || c == '\t'; }

/* getWordFromString: the next word of `line` from *idx (runs of spaces and
 * tabs separate words); returns 0 at the end of the line.  *eol is set when
 * the word ends the line. */
static int next_word(const char *line, size_t *idx, const char **w, size_t *wlen, int *eol)
{
    size_t i = *idx;
    *eol = 0;
    while (is_sep(line[i]))
        ++i;
    if (line[i] == '\0') {
        *eol = 1;
        *idx = i;
        return 0;
    }
    const size_t s = i;
    while (line[i] != '\0' && !is_sep(line[i]))
        ++i;
    *w = line + s;
    *wlen = i - s;
    if (line[i] == '\0')
        *eol = 1;
    *idx = line[i] == '\0' ? i : i + 1;
    return 1;
}

static int valid_base(char c)
{
    return c == 'A' || c == 'C' || c == 'G' || c == 'T' || c == 'N' || c == 'a' || c == 'c' ||
           c == 'g' || c == 't' || c == 'n' || c == '.';
}

/* gz file (or plain text) -> NUL-terminated buffer. */
static char *read_all(const char *path, size_t *bytes)
{
    gzFile f = gzopen(path, "rb");
    if (!f)
        return NULL;
    gzbuffer(f, 1 << 20);
    size_t cap = 1 << 22, len = 0;
    char *buf = malloc(cap + 1);
    while (buf) {
        if (len == cap) {
            char *nb = realloc(buf, cap * 2 + 1);
            if (!nb) {
                free(buf);
                buf = NULL;
                break;
            }
            buf = nb;
            cap *= 2;
        }
        const size_t want = cap - len > (1u << 30) ? (1u << 30) : cap - len;
        const int n = gzread(f, buf + len, (unsigned)want);
        if (n < 0) {
            free(buf);
            buf = NULL;
            break;
        }
        if (n == 0)
            break;
        len += (size_t)n;
    }
    gzclose(f);
    if (buf) {
        buf[len] = '\0';
        *bytes = len;
    }
    return buf;
}

/* getNextLine: the next line of text[*at..end) without its '\n'; lines of
 * fewer than 3 characters give 0 ("no line"), the end of text gives -1. */
static int next_line(char *text, size_t end, size_t *at, char **line)
{
    if (*at >= end)
        return -1;
    char *s = text + *at;
    char *nl = memchr(s, '\n', end - *at);
    if (nl) {
        *nl = '\0';
        *at = (size_t)(nl - text) + 1;
    } else {
        *at = end;
    }
    *line = s;
    return strlen(s) >= 3 ? 1 : 0;
}

void qld_vcf_header_free(qld_vcf_header *h)
{
    if (!h)
        return;
    free(h->line1);
    free(h->line2);
    free(h->valid);
    memset(h, 0, sizeof *h);
}

int qld_vcf_read_header(const char *dir, int ploidy, const char *const *sample_list, int nlist,
                        qld_vcf_header *h)
{
    if (!dir || !h || ploidy < 1)
        return qld_host_fail(QLD_ERR_INVALID, "bad arguments");
    memset(h, 0, sizeof *h);
    DIR *dp = opendir(dir);
    if (!dp)
        return qld_host_fail(QLD_ERR_INVALID, "cannot open directory %s", dir);
    struct dirent *e;
    char name[1024] = "";
    while ((e = readdir(dp))) {   /* the first header file in directory order */
        char path[4096];
        struct stat st;
        snprintf(path, sizeof path, "%s/%s", dir, e->d_name);
        if (stat(path, &st) == 0 && S_ISREG(st.st_mode) && strstr(e->d_name, "header")) {
            snprintf(name, sizeof name, "%s", e->d_name);
            break;
        }
    }
    closedir(dp);
    if (!name[0])
        return qld_host_fail(QLD_ERR_INVALID, "Could not find Header file in %s", dir);
    const size_t k = strcspn(name, "_'");
    if (k == 0 || k >= sizeof h->id)
        return qld_host_fail(QLD_ERR_INVALID, "bad header file name %s", name);
    memcpy(h->id, name, k);
    h->id[k] = '\0';
    snprintf(h->path, sizeof h->path, "%s/%s", dir, name);
    size_t bytes = 0;
    char *text = read_all(h->path, &bytes);
    if (!text)
        return qld_host_fail(QLD_ERR_INVALID, "cannot read %s", h->path);
    size_t at = 0;
    char *line;
    int rc = QLD_OK, st;
    if ((st = next_line(text, bytes, &at, &line)) != 1) {
        rc = qld_host_fail(QLD_ERR_INVALID, "%s: empty header file", h->path);
        goto out;
    }
    h->line1 = strdup(line);
    while ((st = next_line(text, bytes, &at, &line)) != -1) {
        if (st != 1 || strncmp(line, "#CHROM", 6) != 0)
            continue;
        h->line2 = strdup(line);
        size_t idx = 0, wl;
        const char *w;
        int eol, nf = 0;
        while (nf < 9 && next_word(line, &idx, &w, &wl, &eol)) {
            if (wl != strlen(kFixed[nf]) || strncmp(w, kFixed[nf], wl) != 0) {
                rc = qld_host_fail(QLD_ERR_INVALID, "VCF header field %s is missing", kFixed[nf]);
                goto out;
            }
            ++nf;
            if (nf < 9 && eol) {
                rc = qld_host_fail(QLD_ERR_INVALID, "%s: #CHROM line ends early", h->path);
                goto out;
            }
        }
        if (nf < 9) {
            rc = qld_host_fail(QLD_ERR_INVALID, "VCF header field %s is missing", kFixed[nf]);
            goto out;
        }
        int cap = 1024;
        h->valid = malloc((size_t)cap);
        while (h->valid && next_word(line, &idx, &w, &wl, &eol)) {
            if (h->nsamples == cap) {
                uint8_t *nv = realloc(h->valid, (size_t)cap * 2);
                if (!nv)
                    break;
                h->valid = nv;
                cap *= 2;
            }
            int ok = nlist <= 0;
            for (int i = 0; !ok && i < nlist; ++i)
                ok = strlen(sample_list[i]) == wl && strncmp(sample_list[i], w, wl) == 0;
            h->valid[h->nsamples++] = (uint8_t)ok;
            h->valid_count += ok ? ploidy : 0;
            if (eol)
                break;
        }
        if (!h->valid || h->nsamples == 0) {
            rc = qld_host_fail(QLD_ERR_INVALID, "%s: no samples on the #CHROM line", h->path);
            goto out;
        }
        if (next_line(text, bytes, &at, &line) != 1) {
            rc = qld_host_fail(QLD_ERR_INVALID, "Wrong header format");
            goto out;
        }
        char id2[1024];
        if (sscanf(line, "%1023s %d %d %d", id2, &h->snips_per_file, &h->snip_size,
                   &h->total_snips) < 1 ||
            strcmp(id2, h->id) != 0) {
            rc = qld_host_fail(QLD_ERR_INVALID, "Different internal and external ID: %s != %s",
                               id2, h->id);
            goto out;
        }
        break;
    }
    if (rc == QLD_OK && !h->line2)
        rc = qld_host_fail(QLD_ERR_INVALID, "%s: no #CHROM line", h->path);
out:
    free(text);
    if (rc != QLD_OK)
        qld_vcf_header_free(h);
    return rc;
}

static int first_number(const char *path)
{
    const char *b = strrchr(path, '/');
    b = b ? b + 1 : path;
    int v = 0;
    if (sscanf(b, "%*[^_]_%d", &v) != 1)
        v = 0;
    return v;
}

static int part_order(const void *a, const void *b)
{
    const int x = first_number(*(char *const *)a), y = first_number(*(char *const *)b);
    return (x > y) - (x < y);
}

int qld_vcf_list_parts(const char *dir, const qld_vcf_header *h, char ***paths, int *n)
{
    if (!dir || !h || !paths || !n)
        return qld_host_fail(QLD_ERR_INVALID, "bad arguments");
    *paths = NULL;
    *n = 0;
    DIR *dp = opendir(dir);
    if (!dp)
        return qld_host_fail(QLD_ERR_INVALID, "cannot open directory %s", dir);
    int cap = 0;
    struct dirent *e;
    while ((e = readdir(dp))) {
        char path[4096];
        struct stat st;
        snprintf(path, sizeof path, "%s/%s", dir, e->d_name);
        if (stat(path, &st) || !S_ISREG(st.st_mode) || !strstr(e->d_name, h->id) ||
            strstr(e->d_name, "header") || !strstr(e->d_name, ".vcf.gz"))
            continue;
        const size_t k = strcspn(e->d_name, "_");
        if (k != strlen(h->id) || strncmp(e->d_name, h->id, k) != 0)
            continue;
        if (*n == cap) {
            cap = cap ? cap * 2 : 64;
            char **np = realloc(*paths, sizeof *np * (size_t)cap);
            if (!np)
                break;
            *paths = np;
        }
        (*paths)[(*n)++] = strdup(path);
    }
    closedir(dp);
    if (*n)
        qsort(*paths, (size_t)*n, sizeof **paths, part_order);
    return QLD_OK;
}

void qld_vcf_list_free(char **paths, int n)
{
    for (int i = 0; paths && i < n; ++i)
        free(paths[i]);
    free(paths);
}

/* getValueAF (snip_processing.c:163-241): -1 when the INFO field has no
 * AF; values are read 9 characters at most, a list gives its first value
 * strictly between 0 and 1 (else 0). */
static int info_af(const char *s, size_t len, float *af)
{
    *af = -1.0f;
    if ((len == 1 && s[0] == '.') || len < 4)
        return 0;
    size_t i;
    for (i = 0; i < len - 3; ++i)
        if (s[i] == 'A' && s[i + 1] == 'F' && s[i + 2] == '=' && (i == 0 || s[i - 1] == ';'))
            break;
    if (i == len - 3)
        return 0;
    i += 3;
    char v[10] = "";
    float freqs[1000];
    int k = 0;
    for (int j = 0; j < 9; ++j) {
        if (i < len && s[i] == ',') {
            if (!v[0] || k >= 998)
                return qld_host_fail(QLD_ERR_INVALID, "bad AF list in INFO");
            freqs[k++] = (float)atof(v);
            j = 0;
            ++i;
        }
        if (i >= len || s[i] == ';')
            break;
        const char c = s[i];
        if (c == '.' || (c >= '0' && c <= '9') || c == 'e' || c == '-' || c == '+') {
            v[j] = c;
            v[j + 1] = '\0';
            ++i;
        } else {
            return qld_host_fail(QLD_ERR_INVALID, "Invalid character (%c) in AF of field INFO",
                                 c);
        }
    }
    if (!v[0])
        return qld_host_fail(QLD_ERR_INVALID, "AF in field INFO has no value");
    float a;
    if (k == 0) {
        a = (float)atof(v);
    } else {
        freqs[k++] = (float)atof(v);
        a = 0.0f;
        for (int q = 0; q < k; ++q)
            if (freqs[q] > 0.0f && freqs[q] < 1.0f) {
                a = freqs[q];
                break;
            }
    }
    if (a < 0.0f || a > 1.0f)
        return qld_host_fail(QLD_ERR_INVALID, "AF (%f) should be >= 0.0 and <= 1.0", a);
    *af = a;
    return 0;
}

/* checkVTisSNP (:243-268): -1 without VT, 1 for VT=SNP, else 0. */
static int info_vt_snp(const char *s, size_t len, int *vt)
{
    *vt = -1;
    if ((len == 1 && s[0] == '.') || len < 4)
        return 0;
    size_t i;
    for (i = 0; i < len - 3; ++i)
        if (s[i] == 'V' && s[i + 1] == 'T' && s[i + 2] == '=' && (i == 0 || s[i - 1] == ';'))
            break;
    if (i == len - 3)
        return 0;
    i += 3;
    if (i > len - 3)
        return qld_host_fail(QLD_ERR_INVALID, "VT value too short in INFO");
    *vt = s[i] == 'S' && s[i + 1] == 'N' && s[i + 2] == 'P';
    return 0;
}

/* getGTpos (:270-304): index of the "GT" subfield of FORMAT, or -1. */
static int gt_pos(const char *s, size_t len)
{
    int p = 0;
    for (size_t i = 0; i + 1 < len; ++i) {
        if (s[i] == ':')
            ++p;
        if (s[i] == 'G' && s[i + 1] == 'T' && (i == 0 || s[i - 1] == ':') &&
            (i + 2 == len || s[i + 2] == ':'))
            return p;
    }
    return -1;
}

void qld_vcf_part_free(qld_ctx *ctx, qld_vcf_part *p)
{
    if (!p)
        return;
    if (p->text && p->pinned)
        qld_cuda_host_free(ctx, p->text);
    else
        free(p->text);
    free(p->sites);
    free(p->pos);
    free(p->ids);
    free(p->id_pool);
    memset(p, 0, sizeof *p);
}

static int grow_sites(qld_vcf_part *out, size_t *cap)
{
    const size_t nc = *cap ? *cap * 2 : 1024;
    qld_vcf_site *ns = realloc(out->sites, sizeof *ns * nc);
    if (ns)
        out->sites = ns;
    uint32_t *np = realloc(out->pos, sizeof *np * nc);
    if (np)
        out->pos = np;
    size_t *ni = realloc(out->ids, sizeof *ni * nc);
    if (ni)
        out->ids = ni;
    if (!ns || !np || !ni)
        return qld_host_fail(QLD_ERR_NOMEM, "out of memory");
    *cap = nc;
    return QLD_OK;
}

int qld_vcf_load_part(qld_ctx *ctx, const char *path, const qld_vcf_header *h,
                      qld_vcf_part *out)
{
    if (!path || !h || !out)
        return qld_host_fail(QLD_ERR_INVALID, "bad arguments");
    memset(out, 0, sizeof *out);
    size_t bytes = 0;
    char *text = read_all(path, &bytes);
    if (!text)
        return qld_host_fail(QLD_ERR_INVALID, "Failed to open file %s", path);
    if (ctx) {   /* the text goes to the GPU: keep it in pinned memory */
        char *pin = NULL;
        if (qld_cuda_host_alloc(ctx, bytes + 1, (void **)&pin) == QLD_OK) {
            memcpy(pin, text, bytes + 1);
            free(text);
            text = pin;
            out->pinned = 1;
        }
    }
    out->text = text;
    out->bytes = bytes;
    size_t at = 0;
    char *line;
    int rc = QLD_OK;
    if (next_line(text, bytes, &at, &line) != 1) {
        rc = qld_host_fail(QLD_ERR_INVALID, "File %s empty", path);
        goto done;
    }
    if (strcmp(line, h->line1) != 0) {
        rc = qld_host_fail(QLD_ERR_INVALID, "%s: Header 1 different", path);
        goto done;
    }
    if (next_line(text, bytes, &at, &line) != 1 || strcmp(line, h->line2) != 0) {
        rc = qld_host_fail(QLD_ERR_INVALID, "%s: Header 2 different", path);
        goto done;
    }
    size_t cap = 0, pool_len = 0, pool_cap = 0;
    int st;
    for (int ln = 3; (st = next_line(text, bytes, &at, &line)) != -1; ++ln) {
        if (st != 1)
            continue;
        ++out->lines;
        /* readTable_x64 reads CHROM and POS first and asserts both exist */
        {
            size_t j = 0, l2;
            const char *w2;
            int e2;
            if (!next_word(line, &j, &w2, &l2, &e2) || !next_word(line, &j, &w2, &l2, &e2)) {
                rc = qld_host_fail(QLD_ERR_INVALID, "%s line %d: no POS field", path, ln);
                goto done;
            }
        }
        size_t idx = 0, wl, idl = 0;
        const char *w, *id = "";
        int eol = 0, pos = -1, skip = 0, gt = -1, nst = 0;
        char states[4] = {'X', 'X', 'X', 'X'};
        for (int el = 0; el < 9 && next_word(line, &idx, &w, &wl, &eol); ++el) {
            switch (el) {
            case 1:
                pos = atoi(w);
                break;
            case 2:
                if (wl >= 256) {
                    rc = qld_host_fail(QLD_ERR_INVALID, "%s line %d: ID longer than 255", path, ln);
                    goto done;
                }
                id = w;
                idl = wl;
                break;
            case 3:   /* REF: one valid base (getStatesREF) */
                if (wl > 1 || w[0] == ',' || w[0] == '<') {
                    skip = 1;
                    break;
                }
                if (!valid_base(w[0])) {
                    rc = qld_host_fail(QLD_ERR_INVALID, "%s line %d: invalid REF %c", path, ln,
                                       w[0]);
                    goto done;
                }
                states[0] = w[0];
                nst = 1;
                break;
            case 4:   /* ALT: one more base; '.' stands for REF (getStatesALT) */
                if (wl > 1 || w[0] == ',' || w[0] == '<') {
                    skip = 1;
                    break;
                }
                if (!valid_base(w[0])) {
                    rc = qld_host_fail(QLD_ERR_INVALID, "%s line %d: invalid ALT %c", path, ln,
                                       w[0]);
                    goto done;
                }
                if (w[0] == states[0]) {
                    rc = qld_host_fail(QLD_ERR_INVALID,
                                       "Nucleotide %c (field ALT) in position %d appears twice "
                                       "(in REF or ALT)", w[0], pos);
                    goto done;
                }
                states[1] = w[0] == '.' ? states[0] : w[0];
                nst = 2;
                break;
            case 6:
                if (!((wl == 4 && !strncmp(w, "PASS", 4)) || (wl == 1 && w[0] == '.')))
                    skip = 1;
                break;
            case 7: {
                if (wl == 1 && w[0] == '.')
                    break;
                /* AF of exactly 0 or 1 skips the line; only then is VT read */
                float af;
                int vt = -1, e;
                char save = w[wl];
                ((char *)w)[wl] = '\0';
                e = info_af(w, wl, &af);
                if (!e && (af == 0.0f || af == 1.0f))
                    skip = 1;
                else if (!e)
                    e = info_vt_snp(w, wl, &vt);
                ((char *)w)[wl] = save;
                if (e) {
                    rc = QLD_ERR_INVALID;
                    goto done;
                }
                if (vt == 0)
                    skip = 1;
                break;
            }
            case 8:
                gt = gt_pos(w, wl);
                if (gt == -1)
                    skip = 1;
                break;
            default:
                break;
            }
            if (skip || eol)
                break;
        }
        if (pos == -1)
            continue;
        if (skip) {
            ++out->skipped;
            continue;
        }
        /* a site: the sample fields are the rest of the line */
        if ((size_t)out->nsites == cap && (rc = grow_sites(out, &cap)) != QLD_OK)
            goto done;
        if (pool_len + idl + 1 > pool_cap) {
            pool_cap = (pool_cap + idl + 1) * 2;
            char *npool = realloc(out->id_pool, pool_cap);
            if (!npool) {
                rc = qld_host_fail(QLD_ERR_NOMEM, "out of memory");
                goto done;
            }
            out->id_pool = npool;
        }
        memcpy(out->id_pool + pool_len, id, idl);
        out->id_pool[pool_len + idl] = '\0';
        qld_vcf_site *s = &out->sites[out->nsites];
        const size_t L = strlen(line);
        const size_t start = eol || idx > L ? L : idx;
        memset(s, 0, sizeof *s);
        s->off = (long long)(line - text) + (long long)start;
        s->len = (int)(L - start);
        s->gt_pos = gt < 0 ? 0 : gt;
        s->n_states = nst;
        memcpy(s->states, states, 4);
        out->pos[out->nsites] = (uint32_t)pos;
        out->ids[out->nsites] = pool_len;
        pool_len += idl + 1;
        ++out->nsites;
    }
done:
    if (rc != QLD_OK)
        qld_vcf_part_free(ctx, out);
    return rc;
}

const char *qld_vcf_site_id(const qld_vcf_part *p, int site)
{
    return p->id_pool + p->ids[site];
}

/* strip_ext (read_file.c:33-45) */
static void strip_ext(char *f)
{
    char *e = f + strlen(f);
    while (e > f && *e != '.' && *e != '\\' && *e != '/')
        --e;
    if (e > f && *e == '.' && e[-1] != '\\' && e[-1] != '/')
        *e = '\0';
}

int qld_mdf_part_path(const char *out_dir, const char *part_path, char *buf, size_t cap)
{
    char tmp[4096];
    snprintf(tmp, sizeof tmp, "%s", part_path);
    strip_ext(tmp);
    strip_ext(tmp);
    const char *b = strrchr(tmp, '/');
    b = b ? b + 1 : tmp;
    const size_t n = strlen(out_dir);
    if (snprintf(buf, cap, "%s%s%s.mdf", out_dir, n && out_dir[n - 1] == '/' ? "" : "/", b) >=
        (int)cap)
        return qld_host_fail(QLD_ERR_INVALID, "output path too long");
    return QLD_OK;
}

int qld_mdf_write_part(const char *path, const char *id, const qld_vcf_part *p, int K,
                       const uint64_t *words, const uint32_t *bc, const uint8_t *keep)
{
    FILE *f = fopen(path, "w");
    if (!f)
        return qld_host_fail(QLD_ERR_INVALID, "Failed to open file %s", path);
    int kept = 0;
    for (int s = 0; s < p->nsites; ++s)
        kept += keep[s] != 0;
    setvbuf(f, NULL, _IOFBF, 1 << 22);
    fprintf(f, "##fileformat=MDFv0.1\n##SNPs:%d\n#CHROM\tPOS\tID\tBC", kept);
    for (int k = 0; k < K; ++k)
        fprintf(f, "\tcompSNP_%d", k);
    char num[24];
    for (int s = 0; s < p->nsites; ++s) {
        if (!keep[s])
            continue;
        fprintf(f, "\n%s\t%d\t%s\t%u", id, (int)p->pos[s], qld_vcf_site_id(p, s), bc[s]);
        const uint64_t *w = words + (size_t)s * K;
        for (int k = 0; k < K; ++k) {   /* "\t%lu" */
            char *e = num + sizeof num;
            uint64_t v = w[k];
            do {
                *--e = (char)('0' + v % 10);
                v /= 10;
            } while (v);
            *--e = '\t';
            fwrite(e, 1, (size_t)(num + sizeof num - e), f);
        }
    }
    return fclose(f) == 0 ? QLD_OK : qld_host_fail(QLD_ERR_INVALID, "write failed: %s", path);
}
