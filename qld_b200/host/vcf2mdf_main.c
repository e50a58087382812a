/*
 * qld-vcf2mdf -- qLD-parse-2MDF on the B200: a qLD-parse-VCF dataset in, MDF
 * parts out, with the genotype fields packed on the GPU (qld_cuda_vcf_pack).
 *
 * Flags are qLD-parse-2MDF's (arg_parser, src/mdf_extension/src/cl_args.c:
 * 22-124): -input DIR, -output DIR (created if missing), -ploidy haploid|
 * phased_diploid|unphased_diploid (default diploid, as qLD's), -sampleList
 * FILE, -seed N; plus -device, -threads (parts decompressed and written in
 * parallel) and -timing.  -impute is refused.  As qLD, the header file is
 * copied into the output directory (io.c:327-330) and every MDF part written
 * is printed.  Unphased genotypes are shuffled with libc rand() seeded as
 * qLD seeds it (srand(N) for -seed N, else the default seed 1), drawn in
 * qLD's order, so the output is qLD's byte for byte.
 */
#define _GNU_SOURCE
#include <errno.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "qld_host.h"

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

typedef struct rng_state {
    unsigned seed;
    int seeded;
} rng_state;

static unsigned draw(void *user)
{
    rng_state *r = user;
    if (!r->seeded) {   /* qLD's process has made no rand() call before its first shuffle */
        srand(r->seed);
        r->seeded = 1;
    }
    return (unsigned)rand();
}

typedef struct job {
    const qld_vcf_header *h;
    char **paths;
    int first, count;
    qld_vcf_part *parts;
    int *rc;
    char (*err)[512];
    /* write stage */
    const char *out_dir;
    int K;
    uint64_t **words;
    uint32_t **bc;
    uint8_t **keep;
    atomic_int next;
} job;

static void *load_worker(void *arg)
{
    job *j = arg;
    for (int i; (i = atomic_fetch_add(&j->next, 1)) < j->count;) {
        j->rc[i] = qld_vcf_load_part(NULL, j->paths[j->first + i], j->h, &j->parts[i]);
        if (j->rc[i])
            snprintf(j->err[i], sizeof j->err[i], "%s", qld_host_last_error());
    }
    return NULL;
}

static void *write_worker(void *arg)
{
    job *j = arg;
    for (int i; (i = atomic_fetch_add(&j->next, 1)) < j->count;) {
        char path[4096];
        j->rc[i] = qld_mdf_part_path(j->out_dir, j->paths[j->first + i], path, sizeof path);
        if (!j->rc[i])
            j->rc[i] = qld_mdf_write_part(path, j->h->id, &j->parts[i], j->K, j->words[i],
                                          j->bc[i], j->keep[i]);
        if (j->rc[i])
            snprintf(j->err[i], sizeof j->err[i], "%s", qld_host_last_error());
    }
    return NULL;
}

static void run_pool(void *(*fn)(void *), job *j, int threads)
{
    atomic_store(&j->next, 0);
    pthread_t tid[64];
    int made = 0;
    for (int t = 1; t < threads && t < 64; ++t)
        if (pthread_create(&tid[made], NULL, fn, j) == 0)
            ++made;
    fn(j);
    for (int t = 0; t < made; ++t)
        pthread_join(tid[t], NULL);
}

static int copy_file(const char *src, const char *dir)
{
    const char *b = strrchr(src, '/');
    b = b ? b + 1 : src;
    char dst[8192];
    snprintf(dst, sizeof dst, "%s/%s", dir, b);
    FILE *in = fopen(src, "rb"), *out = in ? fopen(dst, "wb") : NULL;
    int ok = in && out;
    char buf[1 << 16];
    size_t n;
    while (ok && (n = fread(buf, 1, sizeof buf, in)) > 0)
        ok = fwrite(buf, 1, n, out) == n;
    if (in)
        fclose(in);
    if (out && fclose(out) != 0)
        ok = 0;
    return ok ? 0 : -1;
}

static void usage(FILE *f)
{
    fputs("usage: qld-vcf2mdf -input DIR -output DIR [-ploidy haploid|phased_diploid|"
          "unphased_diploid]\n"
          "                   [-sampleList FILE] [-seed N] [-device D] [-threads T] [-timing]\n",
          f);
}

int main(int argc, char **argv)
{
    const char *in = NULL, *out = NULL, *list_path = NULL;
    int ploidy = 2, device = 0, threads = 8, timing = 0;
    rng_state rng = {1u, 0};
    for (int i = 1; i < argc; ++i) {
        const char *a = argv[i];
        const char *v = i + 1 < argc ? argv[i + 1] : NULL;
        if (!strcmp(a, "-help") || !strcmp(a, "-h") || !strcmp(a, "--help")) {
            usage(stdout);
            return 0;
        }
        if (!strcmp(a, "-timing")) { timing = 1; continue; }
        if (!strcmp(a, "-impute")) {
            fprintf(stderr, "ERROR: -impute is not supported by qld-vcf2mdf\n");
            return 1;
        }
        if (!strcmp(a, "-input") || !strcmp(a, "-output") || !strcmp(a, "-ploidy") ||
            !strcmp(a, "-sampleList") || !strcmp(a, "-seed") || !strcmp(a, "-device") ||
            !strcmp(a, "-threads")) {
            if (!v) {
                fprintf(stderr, "ERROR: %s needs a value\n", a);
                return 1;
            }
            ++i;
            if (!strcmp(a, "-input")) in = v;
            else if (!strcmp(a, "-output")) out = v;
            else if (!strcmp(a, "-sampleList")) list_path = v;
            else if (!strcmp(a, "-seed")) rng.seed = (unsigned)atoi(v);
            else if (!strcmp(a, "-device")) device = atoi(v);
            else if (!strcmp(a, "-threads")) threads = atoi(v) < 1 ? 1 : atoi(v);
            else if (!strcmp(v, "haploid")) ploidy = 1;
            else if (!strcmp(v, "phased_diploid") || !strcmp(v, "unphased_diploid")) ploidy = 2;
            continue;
        }
        /* qLD-parse-2MDF ignores arguments it does not know */
    }
    if (!in) {
        fprintf(stderr, "ERROR: Please specify input file with \"-input\"\n");
        return 1;
    }
    if (!out) {
        fprintf(stderr, "ERROR: Please specify output file with \"-output\"\n");
        return 1;
    }
    struct stat st;
    if (stat(in, &st) || !S_ISDIR(st.st_mode)) {
        fprintf(stderr, "ERROR: Input directory \"%s\" does not exist\n", in);
        return 1;
    }
    if (stat(out, &st) && mkdir(out, 0700) && errno != EEXIST) {
        fprintf(stderr, "ERROR: cannot create %s\n", out);
        return 1;
    }
    /* sample list: whitespace-separated names (getFilter, io.c:104-128) */
    char **names = NULL;
    int nnames = 0;
    if (list_path) {
        FILE *f = fopen(list_path, "r");
        if (!f) {
            fprintf(stderr, "ERROR: Sample List file \"%s\" doesn't exist\n", list_path);
            return 1;
        }
        char word[1024];
        while (fscanf(f, "%1023s", word) == 1) {
            char **nn = realloc(names, sizeof *nn * (size_t)(nnames + 1));
            if (!nn)
                break;
            names = nn;
            names[nnames++] = strdup(word);
        }
        fclose(f);
    }
    const double t0 = now_s();
    qld_vcf_header h;
    if (qld_vcf_read_header(in, ploidy, (const char *const *)names, nnames, &h)) {
        fprintf(stderr, "ERROR: %s\n", qld_host_last_error());
        return 1;
    }
    if (copy_file(h.path, out)) {
        fprintf(stderr, "ERROR: cannot copy %s to %s\n", h.path, out);
        return 1;
    }
    const int K = (h.valid_count + 63) / 64;
    if (K < 1) {
        fprintf(stderr, "ERROR: no valid samples\n");
        return 1;
    }
    char **paths;
    int nparts;
    if (qld_vcf_list_parts(in, &h, &paths, &nparts)) {
        fprintf(stderr, "ERROR: %s\n", qld_host_last_error());
        return 1;
    }
    qld_ctx *ctx = NULL;
    if (qld_cuda_init(device, &ctx) != QLD_OK) {
        fprintf(stderr, "ERROR: no usable CUDA device %d\n", device);
        return 1;
    }
    const double t_init = now_s();
    double load_s = 0, pack_s = 0, write_s = 0;
    long long sites_total = 0, kept_total = 0;
    int status = 0, snip_size = -1;
    const int batch = threads;
    qld_vcf_part *parts = calloc((size_t)batch, sizeof *parts);
    int *rc = calloc((size_t)batch, sizeof *rc);
    char (*err)[512] = calloc((size_t)batch, sizeof *err);
    uint64_t **words = calloc((size_t)batch, sizeof *words);
    uint32_t **bc = calloc((size_t)batch, sizeof *bc);
    uint8_t **keep = calloc((size_t)batch, sizeof *keep);
    for (int p0 = 0; !status && p0 < nparts; p0 += batch) {
        const int cnt = nparts - p0 < batch ? nparts - p0 : batch;
        job j = {&h, paths, p0, cnt, parts, rc, err, out, K, words, bc, keep, 0};
        double t = now_s();
        run_pool(load_worker, &j, threads);
        load_s += now_s() - t;
        t = now_s();
        for (int i = 0; i < cnt && !status; ++i) {
            if (rc[i]) {
                fprintf(stderr, "ERROR: %s\n", err[i]);
                status = 1;
                break;
            }
            qld_vcf_part *p = &parts[i];
            const size_t ns = (size_t)(p->nsites ? p->nsites : 1);
            int *len = malloc(sizeof *len * ns);
            words[i] = malloc(sizeof **words * ns * (size_t)K);
            bc[i] = malloc(sizeof **bc * ns);
            keep[i] = calloc(ns, 1);
            int bad_site = -1;
            if (!len || !words[i] || !bc[i] || !keep[i]) {
                fprintf(stderr, "ERROR: out of memory\n");
                status = 1;
            } else if (qld_cuda_vcf_pack(ctx, p->text, p->bytes, p->sites, p->nsites, h.valid,
                                         h.nsamples, ploidy, K, draw, &rng, words[i], bc[i], len,
                                         keep[i], &bad_site) != QLD_OK) {
                fprintf(stderr, "ERROR: %s%s%s (position %d): %s\n", paths[p0 + i],
                        bad_site >= 0 ? " " : "", bad_site >= 0 ? qld_vcf_site_id(p, bad_site) : "",
                        bad_site >= 0 ? (int)p->pos[bad_site] : -1, qld_cuda_last_error(ctx));
                status = 1;
            } else {
                /* qLD fixes the row length at its first kept site; every later
                 * line must have it (process_data.c:185-198) */
                for (int s = 0; s < p->nsites; ++s) {
                    if (snip_size >= 0 && len[s] != snip_size) {
                        fprintf(stderr, "ERROR: There are %d nucleotides in position %d. "
                                        "Expected %d.\n", len[s], (int)p->pos[s], snip_size);
                        status = 1;
                        break;
                    }
                    if (snip_size < 0 && keep[i][s])
                        snip_size = len[s];
                    kept_total += keep[i][s] != 0;
                }
                sites_total += p->nsites;
            }
            free(len);
        }
        pack_s += now_s() - t;
        if (!status) {
            t = now_s();
            run_pool(write_worker, &j, threads);
            write_s += now_s() - t;
            for (int i = 0; i < cnt; ++i) {
                if (rc[i]) {
                    fprintf(stderr, "ERROR: %s\n", err[i]);
                    status = 1;
                    break;
                }
                char path[4096];
                qld_mdf_part_path(out, paths[p0 + i], path, sizeof path);
                printf("%s\n", path);
            }
        }
        for (int i = 0; i < cnt; ++i) {
            qld_vcf_part_free(NULL, &parts[i]);
            free(words[i]);
            free(bc[i]);
            free(keep[i]);
            words[i] = NULL;
            bc[i] = NULL;
            keep[i] = NULL;
        }
    }
    if (timing)
        fprintf(stderr,
                "{\"parts\": %d, \"sites\": %lld, \"kept\": %lld, \"K\": %d, \"init_s\": %.6f, "
                "\"load_s\": %.6f, \"pack_s\": %.6f, \"write_s\": %.6f, \"total_s\": %.6f}\n",
                nparts, sites_total, kept_total, K, t_init - t0, load_s, pack_s, write_s,
                now_s() - t0);
    free(parts);
    free(rc);
    free(err);
    free(words);
    free(bc);
    free(keep);
    qld_vcf_list_free(paths, nparts);
    qld_vcf_header_free(&h);
    for (int i = 0; i < nnames; ++i)
        free(names[i]);
    free(names);
    qld_cuda_release(ctx);
    return status;
}
