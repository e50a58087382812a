/*
 * qld-ld -- qLD-compute's -mdf workflow on the B200: read MDF datasets into
 * pinned memory (mdf_loader.c), compute the task's r^2 block on the GPU
 * (qld_cuda_ld) and write qLD's report (report.c).
 *
 * Flags are qLD-compute's (commandLineParser, src/correlator/src/
 * correlate_our_kernel.c:146-470) for the parts this path covers: -input,
 * -input2, -inputList, -output, -ploidy, -mdf, -posWmin1/-posWmax1/
 * -posWmin2/-posWmax2, -r2limit, -threads; plus -device, -r2mode
 * reference|exact (default reference: the report is byte-identical to
 * qLD-compute's), -filter gpu|host (default gpu: qld_cuda_ld_hits keeps the
 * report's pairs on the device and only they cross PCIe; host: the dense r^2
 * array comes back and report.c filters it), -countstates (the COUNTSTATES
 * report of qLD-compute's -DCOUNTSTATES build, correlate_IO.c:430-516,
 * instead of r^2) and -timing (per-task phase times as JSON on stderr).
 * -competing, -sorted, -rTable and -gpu are accepted and change nothing
 * (scheduling switches); -seed is rejected as qLD-compute rejects it (its
 * parser falls through to the invalid-parameter error,
 * correlate_our_kernel.c:387-392,434-436).
 * -sampleList FILE / -sampleList2 FILE (correlate_our_kernel.c:260-289):
 * whitespace-separated sample names (getFilter, correlate_IO.c:35-58).  With
 * MDF input qLD-compute uses a list only to size the rows: K =
 * ceil(listed names on the #CHROM line x ploidy / 64) words
 * (correlate_function.c:112-122), of which writeMDF_x64() keeps the first K
 * words of every row (the words of the first samples, not the listed ones:
 * MDF rows are already packed), with the file's BC and the header's
 * snipSize as S.  qld-ld does the same, so its reports stay byte-identical.
 * Table B takes K from -sampleList2 when it comes from -input2 (and K from
 * -sampleList when it is a second window of -input, as qLD-compute reads it
 * with table A's compSize); a K of table B that differs from table A's is
 * refused, where qLD-compute would read table A with table B's stride.
 * Window resolution is preprocess_data()'s (load_balancer.c:122-345), the
 * single-region / two-table choice and the "input2 equals input" rule are
 * correlate_function()'s (correlate_function.c:94-104,239-295), and
 * -inputList tasks are create_task_queue()'s (input_list.c:205-310), written
 * to <output without extension>_<line>.txt.  While the GPU computes one task,
 * a second thread already loads the next.
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include "qld_host.h"

typedef struct task {
    char in1[4096], in2[4096], out[4096];
    int in2set, w1set, w2set;
    int wmin1, wmax1, wmin2, wmax2;
} task;

typedef struct loaded {
    int rc;
    char err[512];
    int single;          /* one table, SYRK-style */
    int tri;             /* report prints j > i (posWset2 == 0) */
    int S, K;
    qld_table A, B;
    double load_s;
} loaded;

/* -sampleList / -sampleList2 names (no list: every sample counts). */
static char **g_list[2];
static int g_nlist[2];

static int read_sample_list(const char *path, int which)
{
    FILE *f = fopen(path, "r");
    if (!f) {
        fprintf(stderr, "ERROR: cannot open sample list %s\n", path);
        return 1;
    }
    char word[4096];
    int cap = 0;
    while (fscanf(f, "%4095s", word) == 1) {
        if (g_nlist[which] == cap) {
            cap = cap ? 2 * cap : 64;
            char **nl = realloc(g_list[which], sizeof *nl * (size_t)cap);
            if (!nl) {
                fclose(f);
                return 1;
            }
            g_list[which] = nl;
        }
        g_list[which][g_nlist[which]++] = strdup(word);
    }
    fclose(f);
    return 0;
}

/* Words per row for a dataset: ceil(valid samples / 64), the valid count
 * being the header's names that the list holds, times the ploidy. */
static int words_for(const char *dir, int which, int ploidy, int *K)
{
    int listed = 0;
    int rc = qld_mdf_listed_samples(dir, (const char *const *)g_list[which], g_nlist[which],
                                    &listed);
    if (rc)
        return rc;
    const long valid = (long)listed * ploidy;
    *K = (int)((valid + 63) / 64);
    return QLD_OK;
}

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static void usage(FILE *f)
{
    fputs("usage: qld-ld -input DIR [-input2 DIR] -output FILE -ploidy haploid|phased_diploid|"
          "unphased_diploid -mdf\n"
          "              [-posWmin1 P -posWmax1 P -posWmin2 P -posWmax2 P] [-inputList CSV]\n"
          "              [-r2limit R] [-threads T] [-device D] [-r2mode reference|exact]\n"
          "              [-sampleList FILE] [-sampleList2 FILE]\n"
          "              [-filter gpu|host] [-countstates] [-timing]\n",
          f);
}

/* getDir(): a directory path with one trailing '/' */
static void as_dir(char *dst, const char *src)
{
    snprintf(dst, 4096, "%s", src);
    size_t n = strlen(dst);
    if (n && dst[n - 1] != '/' && n + 1 < 4096) {
        dst[n] = '/';
        dst[n + 1] = '\0';
    }
}

/* strip_ext() (input_list.c:28-40): drop the last extension of the file name */
static void strip_ext(char *f)
{
    char *e = f + strlen(f);
    while (e > f && *e != '.' && *e != '\\' && *e != '/')
        --e;
    if (e > f && *e == '.' && e[-1] != '\\' && e[-1] != '/')
        *e = '\0';
}

/* Clamp the windows to the headers' ranges and apply qLD's rules
 * (preprocess_data, load_balancer.c:199-268). */
static void resolve_windows(task *t, const qld_mdf_header *h1, const qld_mdf_header *h2)
{
    const int lo1 = h1->pos_min, hi1 = h1->pos_max;
    if (t->w1set) {
        if (t->wmin1 < lo1 || t->wmin1 > hi1)
            t->wmin1 = lo1;
        if (t->wmax1 < lo1 || t->wmax1 > hi1)
            t->wmax1 = hi1;
        if (t->w2set && t->in2set) {
            if (t->wmin2 < h2->pos_min || t->wmin2 > h2->pos_max)
                t->wmin2 = h2->pos_min;
            if (t->wmax2 < h2->pos_min || t->wmax2 > h2->pos_max)
                t->wmax2 = h2->pos_max;
        } else if (t->w2set) {
            if (t->wmin2 < lo1 || t->wmin2 > hi1)
                t->wmin2 = lo1;
            if (t->wmax2 < lo1 || t->wmax2 > hi1)
                t->wmax2 = hi1;
        } else if (t->in2set) {
            t->w2set = 1;
            t->wmin2 = (t->wmin1 < h2->pos_min || t->wmin1 > h2->pos_max) ? h2->pos_min
                                                                          : t->wmin1;
            t->wmax2 = (t->wmax1 < h2->pos_min || t->wmax1 > h2->pos_max) ? h2->pos_max
                                                                          : t->wmax1;
        } else {
            if (t->wmin2 < lo1 || t->wmin2 > hi1)
                t->wmin2 = lo1;
            if (t->wmax2 < lo1 || t->wmax2 > hi1)
                t->wmax2 = hi1;
        }
    } else {
        t->w1set = 1;
        t->wmin1 = t->wmin2 = lo1;
        t->wmax1 = t->wmax2 = hi1;
    }
    /* qLD's "split-file" rule: two inputs over one window report the triangle */
    if (t->in2set && t->w1set && t->w2set && t->wmin1 == t->wmin2 && t->wmax1 == t->wmax2)
        t->w2set = 0;
}

typedef struct load_arg {
    qld_ctx *ctx;
    task *t;
    int ploidy, threads;
    loaded *out;
} load_arg;

static int load_fail(loaded *l, int rc, const char *msg)
{
    l->rc = rc;
    snprintf(l->err, sizeof l->err, "%s", msg);
    return rc;
}

static void *load_task(void *arg)
{
    load_arg *a = arg;
    task *t = a->t;
    loaded *l = a->out;
    memset(l, 0, sizeof *l);
    const double t0 = now_s();
    qld_mdf_header h1, h2;
    if (qld_mdf_read_header(t->in1, &h1) ||
        (t->in2set ? qld_mdf_read_header(t->in2, &h2) : (h2 = h1, 0))) {
        load_fail(l, QLD_ERR_INVALID, qld_host_last_error());
        return NULL;
    }
    if (t->in2set && h1.snip_size != h2.snip_size) {
        char m[256];
        snprintf(m, sizeof m, "the two inputs have different snip sizes: %d != %d",
                 h1.snip_size, h2.snip_size);
        load_fail(l, QLD_ERR_INVALID, m);
        return NULL;
    }
    resolve_windows(t, &h1, &h2);
    /* correlate_function.c:94-104: the same directory twice is one input */
    if (t->in2set && strcmp(t->in1, t->in2) == 0)
        t->in2set = 0;
    if (words_for(t->in1, 0, a->ploidy, &l->K)) {
        load_fail(l, QLD_ERR_INVALID, qld_host_last_error());
        return NULL;
    }
    l->S = h1.snip_size;
    l->single = !t->w2set && !t->in2set;
    l->tri = !t->w2set;
    if (l->K < 1) {
        load_fail(l, QLD_ERR_INVALID, g_nlist[0] ? "no sample of the list is in the header"
                                                 : "no samples in the header");
        return NULL;
    }
    int rc = qld_mdf_load(a->ctx, t->in1, t->wmin1, t->wmax1, l->K, a->threads, &l->A);
    if (rc == QLD_OK && t->in2set && !t->w2set) {
        /* qLD's split-file rule reads table B with posWset = 0, and
         * readTable_x64() then stops after the first line past each part's
         * two header lines (the do-while condition, correlate_IOx64.c:444):
         * the '#CHROM' column-name line that MDF parts carry, at POS 0, which
         * no clamped window holds.  Table B is empty and the report is its
         * header line alone. */
        l->B.K = l->K;
    } else if (rc == QLD_OK && !l->single) {
        /* table B: input2 with window 2, or input with window 2 */
        int K2 = l->K;
        if (t->in2set && words_for(t->in2, 1, a->ploidy, &K2)) {
            load_fail(l, QLD_ERR_INVALID, qld_host_last_error());
            qld_table_free(a->ctx, &l->A);
            return NULL;
        }
        if (K2 != l->K) {
            char m[256];
            snprintf(m, sizeof m, "the inputs' sample counts differ (%d vs %d words)", l->K, K2);
            load_fail(l, QLD_ERR_INVALID, m);
            qld_table_free(a->ctx, &l->A);
            return NULL;
        }
        rc = qld_mdf_load(a->ctx, t->in2set ? t->in2 : t->in1, t->wmin2, t->wmax2, l->K,
                          a->threads, &l->B);
    }
    if (rc != QLD_OK) {
        load_fail(l, rc, qld_host_last_error());
        qld_table_free(a->ctx, &l->A);
        qld_table_free(a->ctx, &l->B);
        return NULL;
    }
    l->load_s = now_s() - t0;
    return NULL;
}

static int read_list(const char *path, const task *base, task **tasks, int *ntasks)
{
    FILE *f = fopen(path, "r");
    if (!f) {
        fprintf(stderr, "ERROR: Input list file not existing!\n");
        return -1;
    }
    char out[4096];
    snprintf(out, sizeof out, "%s", base->out);
    strip_ext(out);
    char line[16384];
    int cap = 16, n = 0;
    task *ts = malloc(sizeof *ts * (size_t)cap);
    for (int ln = 1; ts && fgets(line, sizeof line, f); ++ln) {
        char in1[4096], s1[64], s2[64], in2[4096], s3[64], s4[64];
        if (sscanf(line, "%4095[^,],%63[^,],%63[^,],%4095[^,],%63[^,],%63[^\n]", in1, s1, s2,
                   in2, s3, s4) != 6) {
            printf("ABORTING: Line %d ---Invalid structure---\n", ln);
            continue;
        }
        task t;
        memset(&t, 0, sizeof t);
        as_dir(t.in1, in1);
        as_dir(t.in2, in2);
        t.wmin1 = atoi(s1);
        t.wmax1 = atoi(s2);
        t.wmin2 = atoi(s3);
        t.wmax2 = atoi(s4);
        if (t.wmin1 >= t.wmax1) {
            printf("ABORTING: Line %d ---posWmin greater than posWmax---\n", ln);
            continue;
        }
        if (t.wmin2 >= t.wmax2) {
            printf("ABORTING: Line %d ---posWmin2 greater than posWmax2---\n", ln);
            continue;
        }
        if (access(t.in1, F_OK) != 0 || access(t.in2, F_OK) != 0) {
            printf("ABORTING: Line %d ---Input files do not exist---\n", ln);
            continue;
        }
        t.in2set = t.w1set = t.w2set = 1;
        snprintf(t.out, sizeof t.out, "%s_%d.txt", out, ln);
        if (n == cap) {
            task *nt = realloc(ts, sizeof *ts * (size_t)cap * 2);
            if (!nt)
                break;
            ts = nt;
            cap *= 2;
        }
        ts[n++] = t;
    }
    fclose(f);
    *tasks = ts;
    *ntasks = n;
    return ts ? 0 : -1;
}

/* Report callback of qld_cuda_ld_hits: append the block's rows. */
typedef struct hits_arg {
    qld_report *rep;
    int host_failed;
    double rep_s;
} hits_arg;

static int on_block(void *user, const qld_hits_block *blk)
{
    hits_arg *h = user;
    const double t0 = now_s();
    const int rc = qld_report_hits(h->rep, blk);
    h->rep_s += now_s() - t0;
    if (rc != QLD_OK)
        h->host_failed = 1;
    return rc;
}

/* The task with the report filter on the GPU: only the kept pairs cross
 * PCIe, and each block is formatted while the GPU computes the next. */
static int run_filtered(qld_ctx *ctx, const loaded *l, const char *out, float r2limit,
                        int threads, double *ld_s, double *rep_s)
{
    const qld_table *A = &l->A, *B = l->single ? &l->A : &l->B;
    FILE *fp = fopen(out, "wb");
    if (!fp) {
        fprintf(stderr, "ERROR: cannot write %s\n", out);
        return 1;
    }
    const double t0 = now_s();
    hits_arg h = {NULL, 0, 0.0};
    int rc = qld_report_open(&h.rep, fp, A, B, l->S, threads);
    if (rc == QLD_OK && A->rows && B->rows)
        rc = qld_cuda_ld_hits(ctx, A->words, A->bc, A->rows, B->words, B->bc, B->rows, l->K, l->S,
                              l->single, l->tri, r2limit, on_block, &h);
    if (rc != QLD_OK)
        fprintf(stderr, "ERROR: %s: %s\n", out,
                (h.host_failed || !h.rep) ? qld_host_last_error() : qld_cuda_last_error(ctx));
    qld_report_close(h.rep);
    if (fclose(fp) != 0)
        rc = QLD_ERR_INVALID;
    *ld_s = now_s() - t0;
    *rep_s = h.rep_s;
    return rc != QLD_OK;
}

/* The task with a dense r^2 array copied back and filtered on the host. */
static int run_dense(qld_ctx *ctx, const loaded *l, const char *out, float r2limit, int threads,
                     double *ld_s, double *rep_s)
{
    const qld_table *A = &l->A, *B = l->single ? &l->A : &l->B;
    const double t0 = now_s();
    float *r2 = NULL;
    const size_t cells = (size_t)A->rows * (size_t)B->rows;
    int rc = cells ? qld_cuda_host_alloc(ctx, cells * sizeof(float), (void **)&r2) : QLD_OK;
    if (rc == QLD_OK && cells)
        rc = qld_cuda_ld(ctx, A->words, A->bc, A->rows, B->words, B->bc, B->rows, l->K, l->S,
                         l->single, r2, NULL);
    *ld_s = now_s() - t0;
    int bad = 0;
    FILE *fp = NULL;
    if (rc != QLD_OK) {
        fprintf(stderr, "ERROR: %s: %s\n", out, qld_cuda_last_error(ctx));
        bad = 1;
    } else if (!(fp = fopen(out, "wb"))) {
        fprintf(stderr, "ERROR: cannot write %s\n", out);
        bad = 1;
    } else {
        const double t1 = now_s();
        if (qld_report_write(fp, A, B, r2, l->S, r2limit, l->tri, threads) != QLD_OK) {
            fprintf(stderr, "ERROR: %s: %s\n", out, qld_host_last_error());
            bad = 1;
        }
        if (fclose(fp) != 0)
            bad = 1;
        *rep_s = now_s() - t1;
    }
    if (r2)
        qld_cuda_host_free(ctx, r2);
    return bad;
}

/* COUNTSTATES task (qLD's -DCOUNTSTATES build): every pair's state value on
 * the GPU, then writeStateCount()'s report. */
static int run_states(qld_ctx *ctx, const loaded *l, const char *out, int threads, double *ld_s,
                      double *rep_s)
{
    const qld_table *A = &l->A, *B = l->single ? &l->A : &l->B;
    const double t0 = now_s();
    uint8_t *st = NULL;
    const size_t cells = (size_t)A->rows * (size_t)B->rows;
    int rc = cells ? qld_cuda_host_alloc(ctx, cells, (void **)&st) : QLD_OK;
    if (rc == QLD_OK && cells)
        rc = qld_cuda_count_states(ctx, A->words, A->rows, B->words, B->rows, l->K, l->single,
                                   st);
    *ld_s = now_s() - t0;
    int bad = 0;
    FILE *fp = NULL;
    if (rc != QLD_OK) {
        fprintf(stderr, "ERROR: %s: %s\n", out, qld_cuda_last_error(ctx));
        bad = 1;
    } else if (!(fp = fopen(out, "wb"))) {
        fprintf(stderr, "ERROR: cannot write %s\n", out);
        bad = 1;
    } else {
        const double t1 = now_s();
        if (qld_report_states(fp, A, B, st, l->tri, threads) != QLD_OK) {
            fprintf(stderr, "ERROR: %s: %s\n", out, qld_host_last_error());
            bad = 1;
        }
        if (fclose(fp) != 0)
            bad = 1;
        *rep_s = now_s() - t1;
    }
    if (st)
        qld_cuda_host_free(ctx, st);
    return bad;
}

int main(int argc, char **argv)
{
    task base;
    memset(&base, 0, sizeof base);
    int ploidy = 0, threads = 1, device = 0, mode = QLD_R2_REFERENCE, timing = 0, mdf = 0;
    int gpu_filter = 1, count_states = 0;
    int have_in = 0, have_out = 0;
    float r2limit = 0.2f;   /* qLD-compute's default */
    const char *list = NULL;
    for (int i = 1; i < argc; ++i) {
        const char *a = argv[i];
        const char *v = i + 1 < argc ? argv[i + 1] : NULL;
        if (!strcmp(a, "-h") || !strcmp(a, "-help") || !strcmp(a, "--help")) {
            usage(stdout);
            return 0;
        }
        if (!strcmp(a, "-mdf")) { mdf = 1; continue; }
        if (!strcmp(a, "-timing")) { timing = 1; continue; }
        if (!strcmp(a, "-countstates")) { count_states = 1; continue; }
        /* qLD-compute's scheduling switches: tasks run in list order on one
         * GPU here, so they change nothing in the reports */
        if (!strcmp(a, "-competing") || !strcmp(a, "-sorted") || !strcmp(a, "-rTable") ||
            !strcmp(a, "-gpu"))
            continue;
        if (!v) {
            fprintf(stderr, "ERROR: %s needs a value\n", a);
            return 1;
        }
        ++i;
        if (!strcmp(a, "-input")) { as_dir(base.in1, v); have_in = 1; }
        else if (!strcmp(a, "-input2")) { as_dir(base.in2, v); base.in2set = 1; }
        else if (!strcmp(a, "-inputList")) list = v;
        else if (!strcmp(a, "-output")) { snprintf(base.out, sizeof base.out, "%s", v); have_out = 1; }
        else if (!strcmp(a, "-posWmin1")) { base.wmin1 = atoi(v); base.w1set = 1; }
        else if (!strcmp(a, "-posWmax1")) { base.wmax1 = atoi(v); base.w1set = 1; }
        else if (!strcmp(a, "-posWmin2")) { base.wmin2 = atoi(v); base.w2set = 1; }
        else if (!strcmp(a, "-posWmax2")) { base.wmax2 = atoi(v); base.w2set = 1; }
        else if (!strcmp(a, "-r2limit")) r2limit = (float)atof(v);
        else if (!strcmp(a, "-sampleList")) { if (read_sample_list(v, 0)) return 1; }
        else if (!strcmp(a, "-sampleList2")) { if (read_sample_list(v, 1)) return 1; }
        else if (!strcmp(a, "-threads")) threads = atoi(v);
        else if (!strcmp(a, "-device")) device = atoi(v);
        else if (!strcmp(a, "-ploidy")) {
            if (!strcmp(v, "haploid")) ploidy = 1;
            else if (!strcmp(v, "phased_diploid") || !strcmp(v, "unphased_diploid")) ploidy = 2;
            else {
                fprintf(stderr, "Please insert supported ploidy (see --help for more info)\n");
                return 1;
            }
        } else if (!strcmp(a, "-filter")) {
            if (!strcmp(v, "gpu")) gpu_filter = 1;
            else if (!strcmp(v, "host")) gpu_filter = 0;
            else {
                fprintf(stderr, "ERROR: -filter is gpu or host\n");
                return 1;
            }
        } else if (!strcmp(a, "-r2mode")) {
            if (!strcmp(v, "reference")) mode = QLD_R2_REFERENCE;
            else if (!strcmp(v, "exact")) mode = QLD_R2_EXACT;
            else {
                fprintf(stderr, "ERROR: -r2mode is reference or exact\n");
                return 1;
            }
        } else {
            fprintf(stderr, "\nERROR: %s is not a valid command line parameter\n\n", a);
            return 1;
        }
    }
    if (!ploidy) {
        fprintf(stderr, "Please insert supported ploidy (see --help for more info)\n");
        return 1;
    }
    if (!mdf) {
        fprintf(stderr, "ERROR: qld-ld reads MDF datasets only: pass -mdf\n");
        return 1;
    }
    if ((!have_in && !list) || !have_out) {
        usage(stderr);
        return 1;
    }
    if (threads < 1)
        threads = 1;

    task *tasks = NULL;
    int ntasks = 0;
    if (list) {
        if (read_list(list, &base, &tasks, &ntasks))
            return 1;
    } else {
        tasks = malloc(sizeof *tasks);
        if (!tasks)
            return 1;
        tasks[0] = base;
        ntasks = 1;
    }

    const double t_init = now_s();
    qld_ctx *ctx = NULL;
    int rc = qld_cuda_init(device, &ctx);
    if (rc != QLD_OK) {
        fprintf(stderr, "ERROR: no usable CUDA device %d: %s\n", device, qld_cuda_last_error(NULL));
        free(tasks);
        return 1;
    }
    qld_cuda_set_option(ctx, QLD_OPT_R2_MODE, mode);
    if (timing)
        fprintf(stderr, "{\"init_s\": %.6f}\n", now_s() - t_init);

    int status = 0;
    loaded cur, next;
    load_arg la = {ctx, &tasks[0], ploidy, threads, &cur};
    if (ntasks)
        load_task(&la);
    for (int t = 0; t < ntasks; ++t) {
        pthread_t pre;
        int prefetching = 0;
        load_arg na = {ctx, t + 1 < ntasks ? &tasks[t + 1] : NULL, ploidy, threads, &next};
        if (t + 1 < ntasks && pthread_create(&pre, NULL, load_task, &na) == 0)
            prefetching = 1;
        if (cur.rc != QLD_OK) {
            fprintf(stderr, "ERROR: %s: %s\n", tasks[t].out, cur.err);
            status = 1;
        } else {
            double ld_s = 0, rep_s = 0;
            const qld_table *B = cur.single ? &cur.A : &cur.B;
            if (count_states ? run_states(ctx, &cur, tasks[t].out, threads, &ld_s, &rep_s)
                             : (gpu_filter ? run_filtered : run_dense)(ctx, &cur, tasks[t].out,
                                                                      r2limit, threads, &ld_s,
                                                                      &rep_s))
                status = 1;
            if (timing)
                fprintf(stderr,
                        "{\"task\": \"%s\", \"rows_a\": %d, \"rows_b\": %d, \"load_s\": %.6f, "
                        "\"ld_s\": %.6f, \"report_s\": %.6f, \"filter\": \"%s\"}\n",
                        tasks[t].out, cur.A.rows, B->rows, cur.load_s, ld_s, rep_s,
                        count_states ? "states" : gpu_filter ? "gpu" : "host");
        }
        qld_table_free(ctx, &cur.A);
        qld_table_free(ctx, &cur.B);
        if (prefetching)
            pthread_join(pre, NULL);
        else if (t + 1 < ntasks)
            load_task(&na);
        cur = next;
    }
    qld_cuda_release(ctx);
    free(tasks);
    return status;
}
