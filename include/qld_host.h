/*
 * qld_host.h -- C host layer of the -cuda mode: MDF dataset loading into
 * pinned memory and the text report, both multithreaded, and the host half
 * of VCF -> MDF conversion (libqld_host.so).
 *
 * Formats are qLD's own:
 *  - an MDF dataset is a directory with <id>_header.vcf.gz (VCF meta line,
 *    #CHROM ... FORMAT <samples> line, then "<id> snipsPerFile snipSize
 *    totalSnips posMin posMax": readHeaderFile, src/correlator/src/
 *    correlate_IO.c:79-259) and parts <id>_<i0>_<i1>_<pos0>_<pos1>.mdf whose
 *    rows are CHROM POS ID BC w0 w1 ... with decimal 64-bit words
 *    (writeMDF_x64 / readTable_x64, correlate_IOx64.c:27-122,351-461);
 *  - the report is writeResultsHeader()/writeResults() (correlate_IO.c:378-429)
 *    with fprint_f()'s 9-digit truncation (fast_print.c:35-103).
 * Status codes are qld_cuda.h's.
 */
#ifndef QLD_HOST_H
#define QLD_HOST_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#include "qld_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qld_mdf_header {
    char id[256];          /* alignment id: the header file name up to its first '_' */
    int snips_per_file;
    int snip_size;         /* S of the r^2 epilogue */
    int total_snips;
    int pos_min, pos_max;
    int samples;           /* sample names on the #CHROM line */
} qld_mdf_header;

/* One region read from a dataset: rows in file order, K words each. */
typedef struct qld_table {
    uint64_t *words;       /* rows x K: pinned (qld_cuda_host_alloc) when loaded with a
                              context, else 64-byte aligned pageable memory */
    uint32_t *bc;          /* the rows' BC field */
    uint32_t *pos;         /* POS */
    char **ids;            /* ID strings */
    char *id_pool;
    int rows, K;
    int pinned;            /* words came from qld_cuda_host_alloc */
} qld_table;

/* Replaces readHeaderFile() (correlate_IO.c:79-259) for an MDF directory. */
int qld_mdf_read_header(const char *dir, qld_mdf_header *h);

/*
 * How many of the sample names on the dataset's #CHROM line appear in
 * `names` (all of them when nnames is 0): makeValidList() + sample_isValid()
 * (correlate_IO.c:60-76,262-290) for a -sampleList read by getFilter()
 * (correlate_IO.c:35-58).  qLD-compute multiplies the result by the ploidy
 * to get the valid sample count that sizes K (correlate_function.c:112-122).
 */
int qld_mdf_listed_samples(const char *dir, const char *const *names, int nnames, int *listed);

/*
 * Rows with pos_min <= POS <= pos_max of every part of the dataset, in file
 * order, K words per row (K = ceil(valid samples / 64)); words past K on a
 * line are ignored, as qLD-compute ignores them (qLD-parse-2MDF's diploid
 * default pads haploid rows with words it does not initialise).  Parts are
 * parsed by `threads` threads and assembled in pinned memory from `ctx`
 * (ctx NULL: pageable memory, no GPU needed).  Replaces findFiles() +
 * readTable_x64() (correlate_IO.c:294-376,
 * correlate_IOx64.c:351-461) for MDF input; returns QLD_ERR_INVALID with a
 * message (qld_host_last_error) for malformed files instead of exiting.
 */
int qld_mdf_load(qld_ctx *ctx, const char *dir, int pos_min, int pos_max, int K, int threads,
                 qld_table *out);
void qld_table_free(qld_ctx *ctx, qld_table *t);   /* ctx: the one it was loaded with */

/*
 * The report of one task: header line, then for B row i (outer) and A row j
 * (inner, j > i for a single region) every r2[i*m + j] with
 * r2limit <= r^2 < 100 as "POS2\tPOS1\tID2\tID1\tfreq[2]\tfreq[1]\tLD".
 * Rows are formatted by `threads` threads and written in order.
 */
int qld_report_write(FILE *fp, const qld_table *A, const qld_table *B, const float *r2,
                     int snip_size, float r2limit, int single_region, int threads);

/*
 * COUNTSTATES report: writeStateCount() (correlate_IO.c:430-470) -- header
 * "POS2\tPOS1\tID2\tID1\tNo_STATES", then for B row i (outer) and A row j
 * (j > i for a single region) "POS2\tPOS1\tID2\tID1\t<states>\t" per line,
 * states[i*m + j] as qld_cuda_count_states() writes them.
 */
int qld_report_states(FILE *fp, const qld_table *A, const qld_table *B, const uint8_t *states,
                      int single_region, int threads);

/*
 * The same report, streamed from qld_cuda_ld_hits blocks: open writes the
 * header line and formats the tables' per-row text once; each call of
 * qld_report_hits appends the rows of one block (blocks in B-row order, as
 * qld_cuda_ld_hits delivers them; it can be called from its callback).
 */
typedef struct qld_report qld_report;
int qld_report_open(qld_report **rep, FILE *fp, const qld_table *A, const qld_table *B,
                    int snip_size, int threads);
int qld_report_hits(qld_report *rep, const qld_hits_block *block);
int qld_report_close(qld_report *rep);

/*
 * VCF -> MDF (qLD-parse-2MDF, src/mdf_extension/src): the host reads a
 * qLD-parse-VCF dataset -- a "*header*" file and parts <id>_<i0>_<i1>_<p0>_
 * <p1>.vcf.gz -- and filters each data line on its fixed fields; the GPU
 * turns the surviving lines' sample fields into packed rows
 * (qld_cuda_vcf_pack); the host writes the MDF parts.
 */
typedef struct qld_vcf_header {
    char id[256];          /* alignment id: the header file name up to '_' */
    char path[4096];       /* the header file (copied next to the MDF parts) */
    char *line1, *line2;   /* the first line and the #CHROM line every part repeats */
    int nsamples;          /* sample names on the #CHROM line */
    uint8_t *valid;        /* per sample: 1 if selected (no sample list: all) */
    int valid_count;       /* selected samples x ploidy: K = ceil(valid_count / 64) */
    int snips_per_file, snip_size, total_snips;
} qld_vcf_header;

int qld_vcf_read_header(const char *dir, int ploidy, const char *const *sample_list, int nlist,
                        qld_vcf_header *h);
void qld_vcf_header_free(qld_vcf_header *h);
/* The dataset's part files in qLD's order (the first number after '_'). */
int qld_vcf_list_parts(const char *dir, const qld_vcf_header *h, char ***paths, int *n);
void qld_vcf_list_free(char **paths, int n);

typedef struct qld_vcf_part {
    char *text;            /* decompressed part (pinned when loaded with a context) */
    size_t bytes;
    int pinned;
    int lines;             /* data lines read */
    int skipped;           /* lines dropped on their fixed fields */
    int nsites;            /* the other lines: sites for qld_cuda_vcf_pack */
    qld_vcf_site *sites;
    uint32_t *pos;         /* per site: POS */
    size_t *ids;           /* per site: offset of its ID in id_pool */
    char *id_pool;
} qld_vcf_part;

int qld_vcf_load_part(qld_ctx *ctx, const char *path, const qld_vcf_header *h,
                      qld_vcf_part *out);
void qld_vcf_part_free(qld_ctx *ctx, qld_vcf_part *p);
const char *qld_vcf_site_id(const qld_vcf_part *p, int site);

/* <out_dir>/<part name without ".vcf.gz">.mdf, and the MDF text of the kept
 * sites (process_data.c:441-460). */
int qld_mdf_part_path(const char *out_dir, const char *part_path, char *buf, size_t cap);
int qld_mdf_write_part(const char *path, const char *id, const qld_vcf_part *p, int K,
                       const uint64_t *words, const uint32_t *bc, const uint8_t *keep);

const char *qld_host_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* QLD_HOST_H */
