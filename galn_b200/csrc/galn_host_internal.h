// galn_host_internal.h -- host-side state shared by galn_host.cpp, galn_engine.cpp and galn_serve.cpp.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/galn_aln.h"
#include "galn_internal.h"

namespace galn {

// a grow-only device or pinned-host buffer
struct Buf {
    void *p = nullptr;
    size_t n = 0;
    bool host = false;
    int ensure(size_t bytes)
    {
        if (bytes <= n) return 0;
        release();
        size_t want = bytes + bytes / 4 + 4096;
        cudaError_t e = host ? cudaMallocHost(&p, want) : cudaMalloc(&p, want);
        if (e != cudaSuccess) { cudaGetLastError(); p = nullptr; n = 0; return -23; }
        n = want;
        return 0;
    }
    void release()
    {
        if (p) { if (host) cudaFreeHost(p); else cudaFree(p); }
        p = nullptr;
        n = 0;
    }
};

// every buffer one search job uses, kept across calls on the same index (calls are serialised)
struct JobBufs {
    Buf seq, query, off, bidx, maxdiff, bopt, out_n, out_off, out_pops, out_trace, out_peak, out_fetch, out_tier,
        out_rec, rec_top, list_a, list_b, counters, ws, dbg, rec_off, rec_ord, tile;
    Buf h_n, h_off, h_pops, h_trace, h_rec, h_list, h_misc, h_res;
    JobBufs()
    {
        h_n.host = h_off.host = h_pops.host = h_trace.host = h_rec.host = h_list.host = h_misc.host = h_res.host = true;
    }
    void release()
    {
        Buf *all[] = {&seq, &query, &off, &bidx, &maxdiff, &bopt, &out_n, &out_off, &out_pops, &out_trace, &out_peak,
                      &out_fetch, &out_tier, &dbg, &out_rec, &rec_top, &list_a, &list_b, &counters, &ws, &rec_off,
                      &rec_ord, &tile, &h_n, &h_off, &h_pops, &h_trace, &h_rec, &h_list, &h_misc, &h_res};
        for (Buf *b : all) b->release();
    }
};

// statistics of the last run (for benchmarks and tests)
struct RunStats {
    double ms_total = 0, ms_kernels = 0, ms_device = 0;
    // host time from the call's start to: the first launch, the device's end, results ready, the first tier's
    // end seen on the host (persistent two-launch form), the warp tier's launch, the first tier's graph launch
    double ms_phase[6] = {0, 0, 0, 0, 0, 0};
    double ms_tier[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int tiers = 0;
    int64_t overflow_reads[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t tier_threads[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t tier_reads[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t kernel_launches = 0;
    int64_t graph_launches = 0;      // of those, launched through a CUDA graph
    uint64_t warp_dbg[16] = {};      // warp-tier counters (keep_stats runs)
    bool fused = false;              // the first tier and the warp tier ran as one launch (ms_tier[0])
    int64_t warp_queued = 0;         // reads the warp tier's first pass queued for its big-arena warps
    int warp_gave_up = 0;            // a big warp's bounded wait ran out in the first pass
    std::vector<uint32_t> fetch;     // per read, of the last run
    std::vector<int8_t> tier_of;     // per read, of the last run
};

// what one search job runs on: a stream, its device buffers and the statistics of its last run
struct ExecCtx {
    cudaStream_t stream = nullptr;
    JobBufs ws;
    RunStats last;
    double mem_share = 1.0;            // of the budget this context's workspace may take
    cudaGraphExec_t graph_exec = nullptr;   // the persistent first-tier launch, captured
    cudaGraphExec_t fused_exec = nullptr;   // the fused launch of the first and warp tiers, captured
    int l2_occ = 0;                    // the layout the stream's persisting L2 window covers (0: none set)
    void release()
    {
        if (graph_exec) { cudaGraphExecDestroy(graph_exec); graph_exec = nullptr; }
        if (fused_exec) { cudaGraphExecDestroy(fused_exec); fused_exec = nullptr; }
        ws.release();
    }
};

}  // namespace galn

struct galn_index {
    galn::DevIndex dev;
    cudaStream_t stream = nullptr;     // the main context's stream
    int sms = 0;
    std::mutex mu;                     // serialises galn_aln_run_batch calls on the main context
    galn::ExecCtx main;
    // tuning knobs (galn_tune.cpp sets them; defaults otherwise)
    int t0_cap = 1024, t0_aln = 32, t0_block = 128;
    int plain_t0_cap = 4096;            // the plain engine's first tier (the reference's light_cap)
    int t1_cap = 65536, t1_aln = 1024;
    double mem_fraction = 0.6;          // of free device memory a job's workspace may take
    bool keep_stats = false;            // keep per-read fetch counts and tiers of the last run
    bool trace = true;                  // compute the per-read trace hash (the reference's --verify data)
    bool use_warp = true;               // the warp tier for reads that overflow T0
    struct TuneChoice { int cap, block, occ, arena, big, fused_div; };
    std::map<uint64_t, TuneChoice> tuned;   // option-set key -> the autotuner's choice
    int occ = 64;                       // occurrence layout when the autotuner has no choice (64 or 80)
    bool tune_active = false;           // the autotuner is timing a candidate: ignore the table
    bool use_graph = true;              // launch the persistent first tier through a CUDA graph
    bool use_fused = false;             // untuned option sets: the first and warp tiers in one launch
    int fused_div = 16;                 // 1 / fused_div of its blocks are warp-tier warps from the start
    int warp_arena = 1 << 13;           // chunks (kWarpChunk entries) per warp
    int warp_big = 128;                 // warps of a warp-tier launch whose arenas hold the max_entries cut-off
    int warp_order = 0;                 // heavy reads' order: 0 max_diff then length, 1 first-tier pops at overflow
    uint64_t warp_wait_ns = 2000000000ull;   // a big warp's bounded wait for queued work
    bool l2_persist = true;             // the occurrence blocks in a persisting L2 window
    bool l2_warm = true;                // and read once through L2 before each search (index_l2_warm)
    // suffix-array samples (<prefix>.sa) for positions; sample 0 is the $ row (-1)
    galn::Buf sa_samples, sa_k, sa_len, sa_pos, sa_strand;
    uint64_t sa_intv = 0, n_sa = 0;
};

namespace galn {
uint64_t opts_key(const galn_opts *o);
// what galn_results._priv owns
// A vector whose resize leaves new elements uninitialised (results are overwritten by a device copy at once).
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U> &) {}
    template <class U>
    void construct(U *p) noexcept { ::new ((void *)p) U; }
    template <class U, class... A>
    void construct(U *p, A &&...a) { ::new ((void *)p) U(std::forward<A>(a)...); }
};
template <class T>
using hvec = std::vector<T, NoInitAlloc<T>>;

struct ResultsPriv {
    hvec<int32_t> n_aln;
    hvec<int64_t> rec_off;
    hvec<galn_aln1> rec;
    hvec<uint64_t> pops, trace;
    void publish(galn_results *out, int n)
    {
        out->n_reads = n;
        out->n_aln = n_aln.data();
        out->rec_offset = rec_off.data();
        out->rec = rec.data();
        out->n_pops = pops.data();
        out->trace = trace.data();
        out->_priv = this;
    }
};
void index_l2_policy(galn_index *ix, cudaStream_t st, int occ);
int index_l2_warm(galn_index *ix, cudaStream_t st, int occ);
void index_l2_clear(galn_index *ix, cudaStream_t st);
int run_job(galn_index *ix, ExecCtx &ctx, const galn_opts *o, const galn_reads *in, int engine, galn_results *out);
int run_job_multi(galn_index *ix, ExecCtx &ctx, const galn_opts *sets, int n_sets, const int32_t *batch_set,
                  const galn_reads *in, int engine, galn_results *out);
}  // namespace galn
