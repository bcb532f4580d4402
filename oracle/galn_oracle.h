/* galn_oracle.h -- test infrastructure: the CPU restatement of the `bwa aln` search used as the parity
 * oracle for the CUDA path. Nothing in the product links this; tests, smoke() and the cpu_baseline leg of
 * bench.py load it through ctypes.
 *
 * It restates, in its own code, what the reference computes on this path:
 *   occurrence counts over BWA's .bwt layout          bwtsearch.h:37-108, bwtgap_hd.h:120-192
 *   bwt_match_exact_alt, bwt_cal_width                bwtgap_hd.h:195-242
 *   the score-bucket LIFO priority stack               bwtgap_hd.h:245-306
 *   gap_shadow, int_log2, bwt_match_gap                bwtgap_hd.h:308-473
 *   the trace hash                                     bwtgap_hd.h:80-100
 *   bwa_cal_maxdiff and the per-batch options          aln_host.c:9-43
 *   FASTQ reading, query encoding and the batch rule   host_io.c:151-215 (kseq.h semantics)
 *   the .sai stream                                    sai_format.h, sai_writer.h
 * The stack grows without bound (upstream's behaviour), so no re-run on overflow is ever needed.
 */
#ifndef GALN_ORACLE_H
#define GALN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* gap_opt_t, the 64-byte option block of the .sai header (field order of bwtaln.h) */
typedef struct {
    int32_t s_mm, s_gapo, s_gape;
    int32_t mode;
    int32_t indel_end_skip, max_del_occ, max_entries;
    float   fnr;
    int32_t max_diff, max_gapo, max_gape;
    int32_t max_seed_diff, seed_len;
    int32_t n_threads;
    int32_t max_top2;
    int32_t trim_qual;
} orc_gap_opt_t;

void *orc_index_load(const char *bwt_path, int *err);
/* the same over a .bwt file image in the caller's memory (not copied; it must outlive the index) */
void *orc_index_borrow(const uint32_t *file_words, uint64_t n_words, int *err);
void  orc_index_free(void *index);
int   orc_index_meta(const void *index, uint64_t *primary, uint64_t L2[5], uint64_t *bwt_words);
/* Occ(c, k) of the four bases at n rows (out[4 i + c]; rows in [0, seq_len] or ~0 for -1) */
void  orc_occ4(const void *index, const uint64_t *rows, int64_t n, uint64_t *out);

void *orc_reads_load(const char *fastq_path, int *n_reads, int64_t *total_bases, int *err);
int   orc_reads_get(const void *reads, uint8_t *query, int64_t *off, int32_t *len, int32_t *batch);
void  orc_reads_free(void *reads);

int   orc_cal_maxdiff(int l, double err, double thres);

void *orc_aln(const void *index, const orc_gap_opt_t *opt, const uint8_t *query, const int64_t *off,
              const int32_t *len, const int32_t *batch, int n_reads, int n_threads);
/* the same with each batch's longest read given for the whole input (these reads may be a shard of it) */
void *orc_aln_bmax(const void *index, const orc_gap_opt_t *opt, const uint8_t *query, const int64_t *off,
                   const int32_t *len, const int32_t *batch, int n_reads, int n_threads, const int32_t *bmax, int n_bmax);
int64_t orc_result_total(const void *res);
int   orc_result_dump(const void *res, int32_t *n_aln, uint64_t *pops, uint64_t *trace, int32_t *peak,
                      uint64_t *fetch128, uint64_t *fetch64, int32_t *n_stacks, int32_t *max_diff,
                      int64_t *rec_off, void *records);
int   orc_result_fetch80(const void *res, uint64_t *fetch80);
/* bwt_sa and bwa_sa2pos over the index and its .sa samples (samples[0] = -1) */
uint64_t orc_bwt_sa(const void *index, const uint64_t *samples, uint64_t intv, uint64_t k);
uint64_t orc_sa2pos(const void *index, const uint64_t *samples, uint64_t intv, uint64_t k, int ref_len, int *strand);
int   orc_result_write_sai(const void *res, const orc_gap_opt_t *opt, const char *path);
/* index files: the suffix array of T$ (sa[0..n], row 0 = position n) by a comparison sort, and <prefix>.bwt
 * / <prefix>.sa for the forward sequence F (codes 0..3) as bwa index writes them (test sizes only) */
int   orc_suffix_array(const uint8_t *T, uint64_t n, uint64_t *sa);
int   orc_index_files(const uint8_t *F, uint64_t l_pac, const char *prefix);
void  orc_result_free(void *res);

#ifdef __cplusplus
}
#endif

#endif
