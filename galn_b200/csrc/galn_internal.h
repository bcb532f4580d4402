// galn_internal.h -- the interface between the host library (galn_host.cpp) and the CUDA code
// (galn_kernels.cu). Not installed; the public interface is include/galn_aln.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "galn_aln.h"

namespace galn {

constexpr int kBatchReads = 0x40000;   // bwa_read_seq batch (src/host_io.h:16)

// per-batch options handed to the device (the layout of BatchOpt in galn_device.cuh)
struct HostBatchOpt {
    int s_mm, s_gapo, s_gape, mode;
    int indel_end_skip, max_del_occ, max_entries;
    int max_diff, max_gapo, max_gape, max_seed_diff, seed_len, max_top2;
    int n_stacks;
    int wide;
    int pad_;
};

struct DevIndex {
    int device = 0;
    uint64_t primary = 0, seq_len = 0, n_blocks = 0;
    uint64_t L2[5] = {0, 0, 0, 0, 0};
    uint64_t sb[16][4] = {};
    void *blocks = nullptr;            // n_blocks * 32 bytes, device (occ64)
    uint64_t n_blocks80 = 0;
    uint64_t sb80[16][4] = {};
    void *blocks80 = nullptr;          // n_blocks80 * 32 bytes, device (occ80)
};

// Builds the occ64 layout on the device from the .bwt body words (host memory).
int dev_index_build(DevIndex &ix, const uint32_t *body, uint64_t n_words, cudaStream_t st);
void dev_index_free(DevIndex &ix);

// Device buffers of one search job (all reads of a request).
struct DevJob {
    int n_reads = 0, n_batches = 0;
    uint8_t *seq = nullptr;            // ASCII, as given
    uint8_t *query = nullptr;          // encoded: reversed+complemented codes
    int64_t *off = nullptr;            // n_reads + 1
    int32_t *bidx = nullptr;           // batch of each read
    int32_t *maxdiff = nullptr;        // per read
    HostBatchOpt *bopt = nullptr;      // per batch (device copy)
    int seed_len = 0;
    int occ = 64;                      // occurrence layout of the kernels (64 or 80 symbols per block)
    int max_len = 0;
    int max_stacks = 0;
    int any_wide = 0;
    int trace = 0;                     // fold every pop into the per-read trace hash
    // outputs, per read
    int32_t *out_n = nullptr;
    int64_t *out_off = nullptr;
    uint64_t *out_pops = nullptr, *out_trace = nullptr;
    int32_t *out_peak = nullptr;
    uint32_t *out_fetch = nullptr;     // 32-byte index blocks read per read (algorithmic traffic)
    int8_t *out_tier = nullptr;        // tier that finished each read
    uint64_t *out_rec = nullptr;       // 3 words per record
    unsigned long long *rec_top = nullptr;
    int64_t rec_cap = 0;
    // work lists
    int32_t *list_a = nullptr, *list_b = nullptr;
    int32_t *counters = nullptr;       // [0] claim, [1] overflow count
};

// Tier parameters of one search launch.
struct TierCfg {
    bool freelist = false;
    int cap = 4096;                    // entries per slot
    int aln_cap = 32;                  // records per slot
    int threads = 0;                   // slots launched
    bool persistent = false;           // claim loop over the list
    int block = 128;
    int tier = 0;
};

struct Workspace;

// Encodes the reads (ASCII -> reversed complemented codes) on the device.
int dev_encode(DevJob &job, cudaStream_t st);

// One coalesced pass over bytes at p through L2 (the stream's access policy applies), one launch.
int dev_l2_warm(const void *p, size_t bytes, int device, cudaStream_t st);

// Launches one search tier over list[0..n) of read ids, appending overflowed reads to ovf[] (count in
// job.counters[1]). ws_mem is a device buffer of at least ws_bytes(cfg, job) bytes.
size_t ws_bytes(const TierCfg &cfg, const DevJob &job);
int dev_search(const DevIndex &ix, DevJob &job, const TierCfg &cfg, const int32_t *list, int n, int32_t *ovf,
               void *ws_mem, cudaStream_t st);

// Occupancy: resident threads per SM for a tier's kernel at the given block size
int dev_resident_threads(const TierCfg &cfg, bool wide, int device);

// The warp tier: one warp per read over list[0..n). Warps 0..n_big-1 have arenas of big_chunks kWarpChunk-entry
// chunks, the others arena_chunks; a read that outgrows a small arena is handed to a big warp in the same
// launch through a queue in ws_mem. Every warp holds aln_cap records. Reads the launch cannot finish go to
// ovf[]; reads still queued when it ends are read back through warp_queue(). ws_mem holds
// warp_ws_bytes(cfg, n) bytes.
// reads the warp tier takes: length and n_stacks (score buckets) at most these; n_stacks is 68-82 for the
// option sets of the benchmark configurations, a read with more goes to the thread tiers
constexpr int kWarpMaxLen = 256, kWarpMaxStacks = 128;
constexpr int kWarpChunk = 64;        // stack entries per chunk of a warp's arena
struct WarpCfg {
    int n_warps = 0, arena_chunks = 0, aln_cap = 0, n_big = 0, big_chunks = 0;
    unsigned long long q_wait_ns = 2000000000ull;   // how long a big warp waits for queued work
};
size_t warp_smem_bytes();
int warp_resident(int device);
size_t warp_ws_bytes(const WarpCfg &c, int n);
constexpr int kWarpDbg = 15;   // counters of the warp tier when profiling is on
int dev_search_warp(const DevIndex &ix, DevJob &job, const WarpCfg &c, int tier, const int32_t *list, int n,
                    int32_t *ovf, void *ws_mem, cudaStream_t st, unsigned long long *dbg);
// The fused launch: the first tier (t0: its slots, cap, records, block of kFusedWarps warps) and the warp tier
// (c: c.n_warps warps in all, n_w_blocks blocks of them warp-tier warps from the start, the big-arena warps
// among those) in one persistent launch; heavy reads pass from the first to the warp tier through a device
// queue. Reads the first tier cannot hand over go to t0_ovf (count in job.counters[1]); reads the warp tier
// cannot finish to the overflow list in FusedQueues (count in job.counters[3]); reads left in the queues are
// read back from FusedQueues (control words: 0 head, 1 tail, 3 a slot was lost).
constexpr int kFusedWarps = 8;
struct FusedQueues {
    int32_t *hq = nullptr, *hq_ctl = nullptr, *w_ovf = nullptr, *q_ctl = nullptr, *big_slots = nullptr;
};
size_t fused_smem_bytes();
int fused_resident_blocks(int device);
size_t fused_ws_bytes(const TierCfg &t0, const DevJob &job, const WarpCfg &c, int n);
void fused_queues(const TierCfg &t0, const DevJob &job, const WarpCfg &c, int n, void *ws_mem, FusedQueues &q);
int dev_search_fused(const DevIndex &ix, DevJob &job, const TierCfg &t0, const WarpCfg &c, int n_w_blocks,
                     const int32_t *list, int n, int32_t *t0_ovf, void *ws_mem, cudaStream_t st, unsigned long long *dbg);
// bwt_sa for n rows d_k (d_ref_len NULL: the forward-reverse coordinate into d_pos) or bwa_sa2pos (with
// d_ref_len: position and strand, ~0 for a hit across the forward/reverse boundary)
int dev_sa_walk(const DevIndex &ix, const uint64_t *d_samples, uint64_t intv, const uint64_t *d_k, int64_t n,
                const int32_t *d_ref_len, uint64_t *d_pos, int8_t *d_strand, cudaStream_t st);
// Occ(c, row) of the four bases at n BWT rows (occ: 4 per row) in layout `occ`, and the blocks read per row
int dev_occ_probe(const DevIndex &ix, int occ, const uint64_t *d_rows, int64_t n, uint64_t *d_occ, uint32_t *d_fetch,
                  cudaStream_t st);
// Results in read order: rec_off[0..n] (exclusive scan of max(out_n, 0)) and the records gathered from
// out_rec into rec_ord; tile_sum holds order_tile_bytes(n) bytes of scratch. Three kernels on st.
int dev_order_results(const DevJob &job, int n, int64_t *rec_off, uint64_t *rec_ord, int64_t *tile_sum, cudaStream_t st);
size_t order_tile_bytes(int n);
// the queue in ws_mem: control words (0 head, 1 tail, 2 small warps finished, 3 a slot was lost) and slots
int32_t *warp_queue(const WarpCfg &c, int n, void *ws_mem, int32_t **slots);
// The device part of `galn index` (galn_build_index.cu): the forward sequence F[0..l_pac) (host, codes
// 0..3) -> the .bwt words after its header (the Occ-interleaved body and the four totals), L2, primary and
// the .sa samples SA[32], SA[64], ...
// Texts of 2^32 - 64 symbols or more, or any text with sort_chunk > 0 (suffixes sorted at once), take the
// builder's 64-bit path.
int dev_build_bwt_sa(const uint8_t *F, uint64_t l_pac, std::vector<uint32_t> &bwt, uint64_t L2[5], uint64_t &primary,
                     std::vector<uint64_t> &samples, galn_build_stats *stats, int64_t sort_chunk = 0);

}  // namespace galn
