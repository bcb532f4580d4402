/* ref_dump.c -- test infrastructure, not product code.
 *
 * A per-read dump harness linked against the reference's own search sources (bwtgap_hd.h,
 * bwtsearch.h, aln_host.c, host_io.c), built by oracle/Makefile into oracle/_ref/libgalnref_dump.so.
 * For every read of a FASTQ it runs the reference's plain host search, aln_search_host
 * (aln_host.c:87-147), with the reference's loader (load_bwt, host_io.c:29-76), FASTQ reader and batch
 * rule (read_fastq / read_batch_ranges, host_io.c:151-215) and per-batch options (aln_batch_opt,
 * aln_read_maxdiff, aln_host.c:23-43), and writes what the reference's --verify check compares
 * (galn.cu:1221-1248): n_aln, the records, n_pops and the trace hash.
 *
 * Dump format (little endian): int64 n_reads; then per read a 40-byte header
 *   int32 n_aln (or a negative error code), int32 batch, int32 len, int32 peak,
 *   uint64 n_pops, uint64 trace, int32 n_stacks, int32 max_diff
 * followed by n_aln 24-byte records (bwt_aln1_t).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include "host_io.h"
#include "aln_host.h"
#include "sai_format.h"

typedef struct {
    int32_t n, batch, len, peak;
    uint64_t pops, trace;
    int32_t n_stacks, max_diff;
} dump_hdr_t;

typedef struct {
    const uint32_t *bwt;
    const bwtgpu_meta_t *meta;
    const uint32_t *cnt;
    const sai_gap_opt_t *opt;
    const bwtgap_opt_t *bopts;
    const int *bstacks;
    const read_t *reads;
    int nreads;
    int next;
    pthread_mutex_t mu;
    dump_hdr_t *hdr;
    bwtgap_aln_t **rec;
} job_t;

static void *work(void *arg)
{
    job_t *J = (job_t*)arg;
    aln_ws_t ws;
    aln_ws_init(&ws);
    for (;;) {
        pthread_mutex_lock(&J->mu);
        int r = J->next++;
        pthread_mutex_unlock(&J->mu);
        if (r >= J->nreads) break;
        int b = J->reads[r].batch;
        int ret = aln_search_host(J->bwt, J->meta, J->cnt, J->opt, &J->bopts[b], J->bstacks[b], &J->reads[r], &ws);
        dump_hdr_t *h = &J->hdr[r];
        h->n = ret; h->batch = b; h->len = J->reads[r].len; h->peak = ws.last_peak;
        h->pops = ws.last_pops; h->trace = ws.last_trace;
        h->n_stacks = J->bstacks[b];
        h->max_diff = aln_read_maxdiff(J->opt, &J->bopts[b], J->reads[r].len);
        if (ret > 0) {
            J->rec[r] = (bwtgap_aln_t*)malloc((size_t)ret * sizeof(bwtgap_aln_t));
            memcpy(J->rec[r], ws.aln, (size_t)ret * sizeof(bwtgap_aln_t));
        }
    }
    aln_ws_free(&ws);
    return NULL;
}

/* opt: a 64-byte sai_gap_opt_t exactly as the reference's parse_args builds it (galn.cu:185-250).
 * Returns the number of reads, or -2 (index), -3 (reads), -5 (output). */
long galnref_dump(const char *bwt_fn, const char *fq_fn, const void *opt_bytes, int nthreads, const char *out_fn)
{
    sai_gap_opt_t opt;
    memcpy(&opt, opt_bytes, sizeof(opt));
    bwtgpu_meta_t meta;
    uint32_t *bwt = load_bwt(bwt_fn, &meta);
    if (!bwt) return -2;
    int nreads = 0;
    read_t *reads = read_fastq(fq_fn, &nreads);
    if (!reads) { free(bwt); return -3; }
    uint32_t cnt[256];
    bwtgap_gen_cnt_table(cnt);
    int *bstart = NULL;
    int nb = read_batch_ranges(reads, nreads, &bstart);
    bwtgap_opt_t *bopts = (bwtgap_opt_t*)calloc(nb > 0 ? nb : 1, sizeof(bwtgap_opt_t));
    int *bstacks = (int*)calloc(nb > 0 ? nb : 1, sizeof(int));
    for (int b = 0; b < nb; ++b)
        bstacks[b] = aln_batch_opt(&opt, reads + bstart[b], bstart[b + 1] - bstart[b], &bopts[b]);
    free(bstart);

    job_t J;
    memset(&J, 0, sizeof(J));
    J.bwt = bwt; J.meta = &meta; J.cnt = cnt; J.opt = &opt; J.bopts = bopts; J.bstacks = bstacks;
    J.reads = reads; J.nreads = nreads;
    J.hdr = (dump_hdr_t*)calloc(nreads > 0 ? nreads : 1, sizeof(dump_hdr_t));
    J.rec = (bwtgap_aln_t**)calloc(nreads > 0 ? nreads : 1, sizeof(bwtgap_aln_t*));
    pthread_mutex_init(&J.mu, NULL);
    if (nthreads < 1) nthreads = 1;
    pthread_t *tid = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    for (int t = 0; t < nthreads; ++t) pthread_create(&tid[t], NULL, work, &J);
    for (int t = 0; t < nthreads; ++t) pthread_join(tid[t], NULL);
    free(tid);

    long ret = nreads;
    FILE *fp = fopen(out_fn, "wb");
    if (!fp) ret = -5;
    else {
        int64_t n64 = nreads;
        fwrite(&n64, 8, 1, fp);
        for (int r = 0; r < nreads; ++r) {
            fwrite(&J.hdr[r], sizeof(dump_hdr_t), 1, fp);
            if (J.hdr[r].n > 0) fwrite(J.rec[r], sizeof(bwtgap_aln_t), (size_t)J.hdr[r].n, fp);
        }
        if (fclose(fp) != 0) ret = -5;
    }
    for (int r = 0; r < nreads; ++r) free(J.rec[r]);
    free(J.rec); free(J.hdr); free(bopts); free(bstacks);
    free_reads(reads, nreads);
    free(bwt);
    return ret;
}

/* size of the option block and of the dump header, for the caller's layout checks */
int galnref_sizes(int *opt_size, int *hdr_size, int *rec_size)
{
    *opt_size = (int)sizeof(sai_gap_opt_t);
    *hdr_size = (int)sizeof(dump_hdr_t);
    *rec_size = (int)sizeof(bwtgap_aln_t);
    return 0;
}
