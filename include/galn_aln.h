/* galn_aln.h -- C ABI of galn-b200, the sm_100a (B200) implementation of the `bwa aln` search.
 *
 * The reference (G-ALN 0.2.7) has no library API: its drop-in surface is the `galn aln` command line, the
 * BWA index files and the .sai stream, and its search is reached internally through
 *     bwtgap_match_gap(bwt, meta, cnt_table, len, seq, width, seed_width, opt, stack, aln, m_aln)
 *         (src/bwtgap_hd.h:338-341, one read)
 *     light_kernel(light_args) / gapw_kernel(gapw_args)  (src/galn.cu:93-135, src/gapw.cuh:86-139, 716-795:
 *         a batch of reads as SoA: query + qoff + qlen, per-read max_diff and batch id, per-batch options)
 * The entry points below replace those seams; each names the reference code it stands in for. All
 * pointers are plain host pointers unless a comment says device; sizes are element counts. No call
 * throws: 0 means success, a negative value is one of the GALN_E* codes.
 *
 * Thread safety: an index handle may be used from several host threads at once; calls on it are
 * serialised internally except galn_aln_submit/galn_aln_wait, which are designed for concurrent use.
 */
#ifndef GALN_ALN_H
#define GALN_ALN_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes (per read, the reference's BWTGAP_ERR_* values, src/bwtgap_hd.h:41-43) ---------- */
#define GALN_OK            0
#define GALN_ERR_STACK   (-1)   /* per read: stack capacity exhausted (internal; the library re-runs) */
#define GALN_ERR_ALN     (-2)   /* per read: record buffer exhausted (internal; the library re-runs) */
#define GALN_ERR_SCORE   (-3)   /* per read: a push scored >= n_stacks (the reference reports it too) */
#define GALN_EINVAL      (-20)  /* bad argument */
#define GALN_EIO         (-21)  /* file missing, short or corrupt */
#define GALN_ECUDA       (-22)  /* CUDA error, or no sm_100 device */
#define GALN_ENOMEM      (-23)  /* host or device allocation failed */
#define GALN_ETIMEOUT    (-24)  /* galn_aln_wait: the request is not finished yet */
#define GALN_EBUSY       (-25)  /* the serving queue is full */

/* ---- options: BWA's gap_opt_t, 64 bytes, written verbatim as the .sai header (src/sai_format.h:16-27) */
typedef struct {
    int32_t s_mm, s_gapo, s_gape;
    int32_t mode;                       /* 0x01 GAPE, 0x02 COMPREAD, 0x04 LOGGAP, 0x10 NONSTOP */
    int32_t indel_end_skip, max_del_occ, max_entries;
    float   fnr;                        /* -n as a fraction, else -1 */
    int32_t max_diff, max_gapo, max_gape;
    int32_t max_seed_diff, seed_len;
    int32_t n_threads;                  /* only the .sai header value (-dt) */
    int32_t max_top2;
    int32_t trim_qual;
} galn_opts;

/* one alignment record, bwt_aln1_t (src/sai_format.h:29-33): packed = n_mm:8 n_gapo:8 n_gape:8
 * score:20 n_ins:10 n_del:10, then the SA interval [k, l] */
typedef struct {
    uint64_t packed, k, l;
} galn_aln1;

/* BWA 0.7.19 defaults (gap_init_opt; the reference's opt_default, src/opt_build.h:23-36) */
int galn_opts_default(galn_opts *o);

/* Parses `galn aln` options (the reference's parse_args, src/galn.cu:185-250): every bwa aln option
 * (-n -o -e -i -d -l -k -m -t/-dt -M -O -E -R -L -N -q0 -f). Positional arguments are returned in
 * pos[0..*n_pos) (at most max_pos), -f in *out_path (or NULL). Returns 0 or GALN_EINVAL (message in err). */
int galn_opts_parse(int argc, const char *const *argv, galn_opts *o, const char **pos, int max_pos, int *n_pos,
                    const char **out_path, char *err, size_t err_len);

/* bwa_cal_maxdiff (src/aln_host.c:9-21): host double arithmetic, no FMA contraction */
int galn_cal_maxdiff(int len, double err, double thres);

/* ---- index ----------------------------------------------------------------------------------------- */
typedef struct galn_index galn_index;

/* Loads <prefix>.bwt (the reference's load_bwt, src/host_io.c:29-76) onto `device` and converts it to
 * the device occurrence layout (32-byte blocks of 64 symbols). The index is read-only afterwards.
 * Returns NULL on error with *err set. */
galn_index *galn_index_open(const char *prefix, int device, int *err);
/* The same from a .bwt already in host memory: the 40-byte header and the body words, as on disk. */
galn_index *galn_index_open_mem(const void *bwt_file_bytes, size_t n_bytes, int device, int *err);
int galn_index_close(galn_index *ix);
/* seq_len (= L2[4]), primary, and the device bytes the occurrence layout takes */
int galn_index_info(const galn_index *ix, uint64_t *seq_len, uint64_t *primary, uint64_t *device_bytes);
/* The occurrence layer on its own: for each of n BWT rows (in [0, seq_len], or ~0 for -1), Occ of the four
 * bases, occ[4 i + c] = bwt_occ4's count (src/bwtgap_hd.h:135-160, src/bwtsearch.h:46-76: the $ row skipped),
 * read from the device layout `layout` (64 or 80 symbols per 32-byte block) by the search's own device code;
 * fetch[i] (may be NULL) the blocks it read. A check of the occurrence layer (no reference counterpart as an
 * entry point); host arrays. */
int galn_index_occ(galn_index *ix, int layout, const uint64_t *rows, int64_t n, uint64_t *occ, uint32_t *fetch);

/* ---- reads ------------------------------------------------------------------------------------------- */
/* A batch of reads as the search takes them: the bases as read (ASCII, any case; A/C/G/T, everything
 * else ambiguous), concatenated, with n_reads+1 offsets. batch[r] is the bwa batch (bwa_read_seq, 0x40000
 * reads, src/host_io.c:164-187) of read r; NULL means consecutive batches of 0x40000 in input order.
 * A batch's options depend on its longest read (src/aln_host.c:23-38): when these reads are a shard of a
 * larger input, batch_max_len[0..n_batches) gives each batch's longest read in the whole input (NULL: the
 * longest among these reads). Reads longer than 65535 bases are rejected (GALN_EINVAL): the reference's
 * stack entry keeps the read position in 16 bits (src/bwtgap_hd.h:365). */
typedef struct {
    int32_t n_reads;
    const char *seq;
    const int64_t *offset;
    const int32_t *batch;
    const int32_t *batch_max_len;
    int32_t n_batches;
} galn_reads;

/* Reads a FASTQ/FASTA file (plain or gzip) with the reference's rules (read_fastq, src/host_io.c:151-205):
 * empty reads skipped, a malformed record dropped and ending its batch. The library owns the memory until
 * galn_read_set_free. */
typedef struct {
    galn_reads reads;
    char **names;
    void *_priv;
} galn_read_set;
int galn_fastq_read(const char *path, galn_read_set *out);
int galn_read_set_free(galn_read_set *rs);

/* The same reader one bwa batch at a time (no reference counterpart; the reference reads batches in a
 * thread of its own, src/galn.cu:580-640): galn_fastq_next fills `out` with the next batch (batch ids as in
 * the whole input; n_reads 0 at the end), freed with galn_read_set_free; the batches of a stream are
 * exactly those galn_fastq_read returns. */
typedef struct galn_fastq_stream galn_fastq_stream;
galn_fastq_stream *galn_fastq_open(const char *path, int *err);
int galn_fastq_next(galn_fastq_stream *s, galn_read_set *out);
int galn_fastq_close(galn_fastq_stream *s);

/* ---- results ------------------------------------------------------------------------------------------ */
/* Per read: n_aln (>= 0, or GALN_ERR_SCORE), records rec[rec_offset[r] .. rec_offset[r+1]) in discovery
 * order (the order the reference writes them), and the instrumentation the reference's --verify compares
 * (n_pops, trace hash; src/galn.cu:1221-1248). Owned by the library until galn_results_free. */
typedef struct {
    int32_t n_reads;
    int32_t *n_aln;
    int64_t *rec_offset;
    galn_aln1 *rec;
    uint64_t *n_pops;
    uint64_t *trace;
    void *_priv;
} galn_results;
int galn_results_free(galn_results *res);

/* ---- search ------------------------------------------------------------------------------------------- */
/* Engines: GALN_ENGINE_PLAIN launches one kernel per bwa batch, one thread per read, and re-runs the reads
 * that overflow their stack in larger tiers (the reference's light tier, src/galn.cu:835-905, with its
 * overflow kept on the GPU). GALN_ENGINE_PERSISTENT runs one persistent work-claiming launch over all
 * batches (captured in a CUDA graph), heavy reads migrating to larger tiers on the device. Both give the
 * same bytes. */
#define GALN_ENGINE_PLAIN       0
#define GALN_ENGINE_PERSISTENT  1

/* Synchronous search of a whole read set (host buffers in, host results out). */
int galn_aln_run_batch(galn_index *ix, const galn_opts *o, const galn_reads *in, int engine, galn_results *out);

/* ---- positions (samse's coordinate step) -----------------------------------------------------------------
 * The next consumer of the .sai records turns a suffix-array row of a hit into a genome position
 * (bwa_cal_pac_pos_core / bwa_sa2pos, src/samse/bwa_upstream/bwase.c:112-139): an LF walk from the row to
 * the nearest sampled row (bwt_sa, bwa's bwt.c:86-96) on the GPU. galn_index_load_sa puts <prefix>.sa on the
 * device (it must belong to the index's .bwt). galn_bwt_sa gives each row's suffix-array value (the
 * forward-reverse coordinate); galn_sa2pos gives bwa_sa2pos's position and strand for a hit of ref_len
 * reference bases (strand 1 = forward, as bwa's !is_rev; position ~0 for a hit across the forward/reverse
 * boundary). Host arrays in and out. */
int galn_index_load_sa(galn_index *ix, const char *prefix);
int galn_bwt_sa(galn_index *ix, const uint64_t *rows, int64_t n, uint64_t *sa);
int galn_sa2pos(galn_index *ix, const uint64_t *rows, const int32_t *ref_len, int64_t n, uint64_t *pos, int8_t *strand);

/* ---- index building (`galn index`) -----------------------------------------------------------------------
 * The files of `bwa index` 0.7.19, byte for byte: <prefix>.pac/.ann/.amb from the FASTA records (the
 * reference's src/index/fasta_pac.c, bwa's bns_fasta2bntseq) and <prefix>.bwt/.sa from the text
 * F . revcomp(F), F the forward sequence with ambiguous bases replaced (the reference's GPU builder,
 * src/index/gpu_index.cu:1-20). The suffix sort, BWT, Occ packing and SA sampling run on the GPU. Texts
 * below 2^32 - 64 symbols (references up to about 2.1 Gbp) take a 32-bit path, about 38 bytes of device
 * memory per symbol; longer ones (a 3.1 Gbp genome is 6.2 x 10^9 symbols) a 64-bit path that sorts in
 * buckets and chunks: 9 bytes per symbol plus 16 per suffix still unsorted after the first 21 symbols, plus
 * the sort buffers (the reference's low-memory builder for such texts is src/index/gpu_sa.cu:1-18). */
typedef struct {
    uint64_t n;                 /* text length, 2 x reference length */
    uint64_t primary;           /* the BWT row of the whole text */
    int rounds;                 /* prefix-doubling rounds after the first sort */
    int sort_passes;            /* 8-bit radix passes, all rounds */
    uint64_t sorted_items;      /* (key, position) pairs sorted, all rounds */
    uint64_t scatter_items;     /* items moved by the radix scatter launches (sorted_items x passes) */
    double ms_device;           /* device time from the text in device memory to the results in device memory */
    double ms_copies;           /* device time of the text's upload and the results' copy back */
    double ms_scatter;          /* device time of the radix scatter launches */
    double ms_files;            /* host time: FASTA to .pac/.ann/.amb, and writing .bwt/.sa */
} galn_build_stats;

/* The host step: <prefix>.pac/.ann/.amb from a FASTA file (plain or gzip), as the reference's
 * galn_fasta_to_pac (src/index/fasta_pac.c:330) writes them; *l_pac = the reference length. FASTQ input is
 * refused (GALN_EINVAL), as is an input without bases. */
int galn_fasta_to_pac(const char *fasta, const char *prefix, uint64_t *l_pac);

/* .bwt and .sa for the forward sequence fwd[0..l_pac) (codes 0..3), built on `device`.
 * Returns 0, GALN_EINVAL (empty or too long), GALN_ENOMEM (device memory), GALN_EIO or GALN_ECUDA.
 * stats may be NULL. */
int galn_index_build_text(const uint8_t *fwd, uint64_t l_pac, const char *prefix, int device, galn_build_stats *stats);
/* The same with the 64-bit path's sort chunk (no reference counterpart): 0 chooses the path by the text's
 * length and the chunk from free device memory; sort_chunk > 0 takes the 64-bit path at any length with at
 * most that many suffixes sorted at once (so small texts exercise its buckets and chunks). The files are
 * the same either way. */
int galn_index_build_text_ex(const uint8_t *fwd, uint64_t l_pac, const char *prefix, int device, int64_t sort_chunk,
                             galn_build_stats *stats);

/* All five files for a FASTA file (plain or gzip), built on `device`, as `galn index -a gpu -p <prefix>
 * <fasta>` writes them (src/index/galn_index.c:36-71). */
int galn_index_build_fasta(const char *fasta, const char *prefix, int device, galn_build_stats *stats);

/* ---- .sai ----------------------------------------------------------------------------------------------- */
/* "SAI\1", the option block, then per read int32 n_aln and the records (src/sai_writer.h:9-21). A read
 * with an error code is written with 0 records and the call returns 4 (src/galn.cu:1250-1263); 5 on a
 * write error. */
int galn_sai_write(const char *path, const galn_opts *o, const galn_results *res);

/* The same stream written in parts (no reference counterpart): open writes the header (path NULL:
 * stdout), each append the reads of one result set in order, close returns what galn_sai_write would
 * (0, 4 or 5). galn_sai_write is open + one append + close. */
typedef struct galn_sai_writer galn_sai_writer;
galn_sai_writer *galn_sai_open(const char *path, const galn_opts *o, int *err);
int galn_sai_append(galn_sai_writer *w, const galn_results *res);
int galn_sai_close(galn_sai_writer *w);

/* ---- serving ---------------------------------------------------------------------------------------------- */
/* A resident index serves requests with their own options and batch boundaries (continuous batching):
 * steps of up to step_reads reads are taken from all admitted requests (equal shares, then oldest first)
 * and searched together; a request that arrives while a step runs joins the next one, and leaves when its
 * last read is done. Requests are admitted by the device memory their search stacks need (galn_stack_need)
 * against a budget of stack_bytes (0: half of the device memory free at start); one that does not fit waits
 * while later requests that fit pass it (at most 64 of them), and is admitted alone at worst. Each
 * request's results are the same bytes as a galn_aln_run_batch of it alone. The reference's equivalent is
 * its per-batch scheduling of one input file with warps and stack arenas sized from free device memory
 * (src/galn.cu:605-635, 835-965). */
typedef struct galn_server galn_server;
galn_server *galn_server_start(galn_index *ix, size_t stack_bytes, int *err);
/* The device memory the server reserves for a request's search stacks while it is admitted (no reference
 * counterpart): a first-tier stack per read of a step (entries, a head per score bucket of its options,
 * the width arrays of its longest read, the records) plus one stack deep enough for its max_entries. */
int galn_stack_need(galn_server *s, const galn_opts *o, const galn_reads *in, uint64_t *bytes);
/* The stack budget, the reservation of the admitted requests now and at most, and how many times a queued
 * request was passed over for lack of stack memory (no reference counterpart). */
int galn_server_memory(galn_server *s, uint64_t *budget, uint64_t *in_use, uint64_t *peak, int64_t *held_back);
/* Up to n request ids in the order they were admitted; returns how many (no reference counterpart). */
int galn_server_admissions(galn_server *s, int64_t *ids, int n);
int galn_server_stop(galn_server *s);
/* copies the request's inputs; returns a request id > 0, or an error */
int64_t galn_aln_submit(galn_server *s, const galn_opts *o, const galn_reads *in);
/* waits up to timeout_ms (-1: forever) for a request; on success moves its results into *out */
int galn_aln_wait(galn_server *s, int64_t id, int timeout_ms, galn_results *out);
/* reads per step (the device workspace of one step) and requests in flight at once (no reference
 * counterpart; defaults 262144 and 64) */
int galn_server_configure(galn_server *s, int step_reads, int max_active);
/* While a step is on the device, start the next only once fill_reads reads (at most a step's worth) are
 * waiting, or when the running step ends (no reference counterpart; 0, the default, starts at once):
 * fuller steps for a caller that submits faster than the device searches, such as a file read batch by
 * batch; results never depend on it. */
int galn_server_set_step_fill(galn_server *s, int fill_reads);
/* submit-to-result latency percentiles of the finished requests, requests and reads finished, device
 * busy milliseconds and steps run (no reference counterpart) */
int galn_server_stats(galn_server *s, double *p50_ms, double *p99_ms, int64_t *n_requests, int64_t *n_reads,
                      double *busy_ms, int64_t *steps);

/* ---- search without device allocation --------------------------------------------------------------
 * No counterpart in the reference. For callers that may not allocate or free device memory while they
 * search (a host framework that owns all GPU memory through its own pool, a stage running under a fixed
 * memory budget, or code that must not trigger the device synchronisation cudaFree implies): the first
 * search tier on reads that already sit in the caller's device buffers, with every byte of scratch taken
 * from one 32 MiB array inside the library (a __device__ array: every GPU that loads the library keeps it
 * until the process exits). Nothing is allocated: no cudaMalloc, cudaFree or allocating library call.
 *   d_seq, d_offset   device: ASCII reads and n_reads+1 offsets; all reads are one bwa batch (at most
 *                     0x40000 reads) whose longest read is max_len (<= 1024 bases)
 *   d_n_aln           device, n_reads: n_aln, GALN_ERR_SCORE, or GALN_ERR_STACK / GALN_ERR_ALN when the read
 *                     needed more than the fixed per-thread stack (2048 entries) or more than rec_per_read
 *                     records (<= 256); such reads can be searched again with galn_aln_run_batch. A read
 *                     longer than max_len (or with offsets out of order) gets GALN_EINVAL and is not searched.
 *   d_rec             device, n_reads * rec_per_read records; read r's at d_rec[r * rec_per_read]
 * Runs asynchronously on `stream` (a cudaStream_t; NULL for the default stream): a memset of the array's
 * work counter and one kernel launch, nothing copied from the host. The first call on a device looks up
 * the array's device address (cudaGetSymbolAddress) and should come before any stream capture. All calls
 * share the array and it keeps the last call's contents: calls that overlap on the GPU (other streams,
 * other host threads) race on it and must be serialised by the caller. The array holds a few hundred
 * per-thread stacks (about 700 for 100-base reads), so this runs far below galn_aln_run_batch's rate.
 * Sizes past the limits above return GALN_EINVAL; options that need more than 512 score buckets or
 * negative penalties too. */
int galn_aln_run_noalloc(galn_index *ix, const galn_opts *o, int32_t n_reads, int32_t max_len, const char *d_seq,
                         const int64_t *d_offset, int32_t *d_n_aln, galn_aln1 *d_rec, int32_t rec_per_read,
                         void *stream);

/* Statistics of the last galn_aln_run_batch on this index (no reference counterpart; the reference prints
 * the same kind of figures with -v, src/galn.cu:1268-1284): wall and kernel milliseconds, tiers used,
 * kernel launches, and the reads that overflowed each tier (8 entries). */
int galn_last_run_stats(galn_index *ix, double *ms_total, double *ms_kernels, int *tiers, int64_t *launches,
                        int64_t *overflow);

/* Device-side profile of the last run (no reference counterpart): the device span from the first to the
 * last kernel (ms); per tier (8 entries each) its kernel ms, the reads it was given and the threads it
 * ran; and, when the index was tuned with keep_stats, per read the 32-byte index blocks read and the tier
 * that finished it (n entries). Any pointer may be NULL. */
int galn_last_run_profile(galn_index *ix, double *ms_device, double *ms_tier, int64_t *tier_reads, int64_t *tier_threads,
                          uint32_t *fetch, int8_t *tier, int32_t n);

/* The autotuner (no reference counterpart): times the first max_sample reads (0: all) once per candidate
 * occurrence layout (64 or 80 symbols per 32-byte block), first-tier stack depth (256..4096 entries: the
 * split between thread-per-read and warp-per-read) and block size, then, with that choice, once per warp-tier
 * arena per warp (8192 or 16384 chunks of 64 entries) and count of big-arena warps (128 or 256), then once per
 * launch form (two launches, or the fused launch with 1/16 .. 1/2 of its blocks warp-tier warps from the
 * start: fused_div 0, or 16 .. 2), and keeps the fastest for this option set; later searches with the same
 * options use it. Returns the first stage's choice and the best device milliseconds; galn_autotune_choice
 * gives the whole choice for an option set (GALN_EINVAL if it has none). galn_autotune_clear forgets all
 * choices. */
int galn_autotune(galn_index *ix, const galn_opts *o, const galn_reads *in, int max_sample, int *best_cap,
                  int *best_block, int *best_occ, double *best_ms);
int galn_autotune_choice(galn_index *ix, const galn_opts *o, int *cap, int *block, int *occ, int *warp_arena,
                         int *warp_big, int *fused_div);
int galn_autotune_clear(galn_index *ix);

/* How many of the last run's kernel launches went through a CUDA graph (no reference counterpart). */
int galn_last_graph_launches(galn_index *ix, int64_t *graph_launches);

/* The persistent engine's first tier and warp tier as one launch (no reference counterpart): blocks of 8
 * warps, as many as stay resident, 1/16 of them warp-tier warps from the start and the others first-tier
 * threads (heaviest reads first) that turn into warp-tier warps when the first tier's reads run out; a read
 * that overflows the first tier is handed to a warp at once through a device queue (the reference's light
 * tier and warp phases hand reads over through its shared list, src/galn.cu:907-1180). This sets the form
 * for option sets the autotuner has not tuned (off by default: two launches); a tuned option set uses the
 * form the autotuner timed fastest. Results never depend on it. galn_last_run_fused tells whether the last
 * run used it (the launch's time is then ms_tier[0] of galn_last_run_profile). */
int galn_index_set_fused(galn_index *ix, int on);
int galn_last_run_fused(galn_index *ix, int *fused);

/* Counters of the warp tier in the last keep_stats run (no reference counterpart): reads searched (with
 * re-runs), waves, entries expanded, entries replayed, pops, chains continued in the next wave, hits, SM
 * cycles in chains / replay / commit / wave loads (summed over warps), pops run (with dropped
 * speculation), SM cycles inside reads, chain steps, the longest read's SM cycles. */
int galn_last_warp_counters(galn_index *ix, uint64_t *counters, int n);

/* Host-side timeline of the last run (no reference counterpart), up to n (<= 8) of: ms from the call's start
 * to the first kernel launch, to the end of the device work, to the results being ready; the call's total
 * ms; the device span in ms; ms from the call's start to the host seeing the first tier's end, to the warp
 * tier's launch and to the first tier's graph launch (0 where the run had no such step). */
int galn_last_run_phases(galn_index *ix, double *ms, int n);

/* Random 32-byte gather peak of the device (no reference counterpart; a measurement for the roofline): the
 * best of `repeats` timed launches of a kernel reading pseudo-random 32-byte sectors of a buffer of the
 * largest power of two <= `bytes` (>= 1 MiB; larger than L2 for the HBM figure, smaller for L2), in GB/s
 * of sectors read. */
int galn_gather_peak(int device, uint64_t bytes, int repeats, double *gbs);
/* The same with in_flight (2, 4, 8 or 16) independent sectors in flight per thread (galn_gather_peak uses 8);
 * 256 sectors per thread, 8 blocks of 256 threads per SM. */
int galn_gather_peak_ex(int device, uint64_t bytes, int in_flight, int repeats, double *gbs);

/* Tier capacities (no reference counterpart; set by the autotuner): entries and records per thread in the
 * first tier, its block size (64/128/256/512), live entries and records per thread in the second tier, and
 * whether to keep the per-read profile. Results never depend on these values. */
int galn_index_set_tuning(galn_index *ix, int t0_cap, int t0_aln, int t0_block, int t1_cap, int t1_aln, int keep_stats);

/* The heavy-read warp tier on or off, and its stack arena per warp in 64-entry chunks (no reference
 * counterpart; on by default with 8192 chunks, at least 32). Results never depend on it. */
int galn_index_set_warp_tier(galn_index *ix, int on, int arena_chunks);

/* How long (ns) a big-arena warp of the warp tier waits for queued reads before it gives up (no reference
 * counterpart; default 2 s). Reads still queued when the warps give up are searched in a second launch, and
 * when a warp gave up on a read id that had not yet arrived in its claimed slot, every read that was ever
 * queued is searched again; results never depend on it. 0 makes every wait run out at once and takes the
 * second of those paths (a way to test it). */
int galn_index_set_warp_wait(galn_index *ix, int64_t wait_ns);
/* The order in which the two-launch form hands the first tier's overflow to the warp tier (no reference
 * counterpart): 0 (default) the largest max_diff, then the longest read first; 1 the reads whose first-tier
 * search overflowed after the fewest pops first. Results never depend on it. */
int galn_index_set_warp_order(galn_index *ix, int order);

/* The last run's warp-tier queues (no reference counterpart): reads its first launch queued for the big-arena
 * warps (and, in the fused launch, from the first tier to the warp tier), and whether a lost queue slot
 * made every queued read be searched again. */
int galn_last_warp_queue(galn_index *ix, int64_t *queued, int *gave_up);

/* The occurrence blocks in a persisting L2 access-policy window on the index's streams (no reference
 * counterpart; on by default; results never depend on it). */
int galn_index_set_l2_persist(galn_index *ix, int on);

/* The occurrence layout the kernels use when the autotuner has no choice for the options (no reference
 * counterpart; 64 by default): 64 or 80 symbols per 32-byte block. The index holds both. Results never
 * depend on it; only the per-read count of blocks read does (it counts blocks of the layout used). */
int galn_index_set_occ_layout(galn_index *ix, int stride);

/* Trace hashes on or off (on by default). The reference computes them only in its --verify mode
 * (gapw_kernel<TRACE>, src/gapw.cuh:716-795); off, the kernels skip the hash and results carry 0 in
 * trace[]. n_aln, records and n_pops are unaffected. */
int galn_index_set_trace(galn_index *ix, int on);

/* library version string */
const char *galn_version(void);

#ifdef __cplusplus
}
#endif

#endif
