// galn_engine.cpp -- one search job on the device: per-batch options, device buffers, and the tiers.
//
// Per-batch options follow the reference's aln_batch_opt / aln_read_maxdiff (src/aln_host.c:23-43): with -n
// as a fraction, a batch's max_diff comes from its longest read and max_gapo is clamped to it; n_stacks =
// score(max_diff+1, max_gapo+1, max_gape+1); each read's max_diff comes from its own length.
//
// Tiers (every read ends on the GPU; there is no CPU fallback):
//   T0   bump-allocated stack of t0_cap entries per thread, t0_aln records: nearly every read ends here
//   T1   free-list stack of t1_cap live entries, t1_aln records, for the reads that overflowed T0
//   T2+  free-list stack of max_entries + 16 live entries (enough to reach the reference's own
//        n_entries > max_entries cut-off exactly), records growing x16 per tier
// A read that overflows is searched again from scratch in the next tier, as the reference re-runs a read
// on overflow (src/aln_host.c:87-147), so results never depend on the capacities.
// PLAIN launches T0 once per bwa batch with one thread per read (the reference's light tier, one launch per
// chunk, src/galn.cu:835-905). PERSISTENT launches T0 once over all reads with as many threads as the
// device keeps resident, each claiming reads from a device counter until none are left.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <numeric>
#include <thread>
#include <unordered_map>
#include <vector>

#include "galn_host_internal.h"

namespace galn {

#define ECK(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            fprintf(stderr, "[galn] CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            return GALN_ECUDA;                                                                \
        }                                                                                     \
    } while (0)
#define RCK(call)                      \
    do {                               \
        int r_ = (call);               \
        if (r_) return r_;             \
    } while (0)

static double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static inline int score_of(int m, int o, int e, const galn_opts *p) { return m * p->s_mm + o * p->s_gapo + e * p->s_gape; }

int run_job(galn_index *ix, ExecCtx &ctx, const galn_opts *o, const galn_reads *in, int engine, galn_results *out)
{
    return run_job_multi(ix, ctx, o, 1, nullptr, in, engine, out);
}

// sets[batch_set[b]] are the options of bwa batch b (all sets[0] when batch_set is NULL)
int run_job_multi(galn_index *ix, ExecCtx &ctx, const galn_opts *sets, int n_sets, const int32_t *batch_set,
                  const galn_reads *in, int engine, galn_results *out)
{
    double t_start = now_ms();
    if (!sets || n_sets < 1) return GALN_EINVAL;
    const int n = in->n_reads;
    if (n < 0 || (n > 0 && (!in->seq || !in->offset))) return GALN_EINVAL;
    JobBufs &B = ctx.ws;
    RunStats &S = ctx.last;
    S = RunStats();
    cudaStream_t st = ctx.stream;
    ECK(cudaSetDevice(ix->dev.device));

    // ---- per-read lengths, batches, options: a few passes over the reads, on several host threads ----
    size_t nn = (size_t)std::max(n, 1);
    RCK(B.h_off.ensure((nn + 1) * 8));
    RCK(B.h_list.ensure(nn * 4 * 4));
    const int64_t total = n > 0 ? in->offset[n] - in->offset[0] : 0;
    const int64_t base = n > 0 ? in->offset[0] : 0;
    // the bases go to the device first, so that the copy runs while the host passes over the reads (a span
    // no valid input can have is left to the checks below)
    if (total > 0 && total <= (int64_t)n * 65535) {
        RCK(B.seq.ensure((size_t)total));
        ECK(cudaMemcpyAsync(B.seq.p, in->seq + base, (size_t)total, cudaMemcpyHostToDevice, st));
    }
    int64_t *h_off = (int64_t *)B.h_off.p;
    // pinned per-read arrays: batch ids, max_diff, the read list (later the first tier's overflow list), and the
    // warp tier's sorted list
    int32_t *h_bid = (int32_t *)B.h_list.p, *h_md = h_bid + nn, *h_list = h_md + nn, *h_wlist = h_list + nn;
    const int32_t *bid = h_bid, *maxdiff = h_md;
    const int T = n >= (1 << 16) ? (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency())) : 1;
    auto par = [&](const std::function<void(int, int, int)> &fn) {
        if (T == 1) { fn(0, n, 0); return; }
        std::vector<std::thread> th;
        for (int t = 0; t < T; ++t)
            th.emplace_back(fn, (int)((int64_t)n * t / T), (int)((int64_t)n * (t + 1) / T), t);
        for (auto &x : th) x.join();
    };
    // pass 1: lengths, batch ids, offsets; per thread the longest read and size of each batch, the lengths seen
    struct Part {
        int max_len = 0;
        bool bad = false, sorted = true;
        std::vector<int> bmax, bcount;
        std::vector<uint8_t> seen;
    };
    std::vector<Part> parts((size_t)T);
    par([&](int r0, int r1, int t) {
        Part &P = parts[(size_t)t];
        P.seen.assign(65536, 0);
        int prev = -1;
        for (int r = r0; r < r1; ++r) {
            const int64_t len = in->offset[r + 1] - in->offset[r];
            const int b = in->batch ? in->batch[r] : r / kBatchReads;
            if (len < 0 || len > 65535 || b < 0) { P.bad = true; return; }
            h_bid[r] = b;
            h_off[r] = in->offset[r] - base;
            if (b < prev) P.sorted = false;
            prev = b;
            if ((size_t)b >= P.bmax.size()) { P.bmax.resize((size_t)b + 1, 0); P.bcount.resize((size_t)b + 1, 0); }
            P.bmax[(size_t)b] = std::max(P.bmax[(size_t)b], (int)len);
            ++P.bcount[(size_t)b];
            P.max_len = std::max(P.max_len, (int)len);
            P.seen[(size_t)len] = 1;
        }
    });
    if (n >= 0) h_off[n] = total;
    int n_batches = 0, max_len = 0;
    bool sorted = true;
    for (int t = 0; t < T; ++t) {
        const Part &P = parts[(size_t)t];
        if (P.bad) return GALN_EINVAL;
        n_batches = std::max(n_batches, (int)P.bmax.size());
        max_len = std::max(max_len, P.max_len);
        sorted = sorted && P.sorted;
        if (t > 0 && sorted) {   // batch ids across the threads' boundary
            const int r = (int)((int64_t)n * t / T);
            if (r > 0 && r < n && h_bid[r] < h_bid[r - 1]) sorted = false;
        }
    }
    // the longest read of each batch: given by the caller when these reads are a shard of a larger input
    if (in->batch_max_len && in->n_batches > n_batches) n_batches = in->n_batches;
    std::vector<int> bmax((size_t)std::max(n_batches, 1), 0), bcount((size_t)std::max(n_batches, 1), 0);
    for (const Part &P : parts)
        for (size_t b = 0; b < P.bmax.size(); ++b) {
            bmax[b] = std::max(bmax[b], P.bmax[b]);
            bcount[b] += P.bcount[b];
        }
    if (in->batch_max_len) {
        if (in->n_batches < n_batches) return GALN_EINVAL;
        for (int b = 0; b < n_batches; ++b) bmax[b] = std::max(bmax[b], (int)in->batch_max_len[b]);
    }
    std::vector<HostBatchOpt> bopt((size_t)std::max(n_batches, 1));
    int max_stacks = 1;
    bool wide = ix->dev.seq_len >= (1ull << 38);
    std::vector<const galn_opts *> bset((size_t)std::max(n_batches, 1), &sets[0]);
    for (int b = 0; b < n_batches; ++b) {
        if (batch_set) {
            if (batch_set[b] < 0 || batch_set[b] >= n_sets) return GALN_EINVAL;
            bset[b] = &sets[batch_set[b]];
        }
    }
    int64_t max_entries_all = 0;
    int seed_part = 0;
    for (int b = 0; b < n_batches; ++b) {
        const galn_opts *o = bset[b];
        max_entries_all = std::max<int64_t>(max_entries_all, o->max_entries);
        if (o->seed_len >= 0 && o->seed_len < max_len) seed_part = std::max(seed_part, o->seed_len);
        HostBatchOpt &h = bopt[b];
        memset(&h, 0, sizeof(h));
        h.s_mm = o->s_mm; h.s_gapo = o->s_gapo; h.s_gape = o->s_gape; h.mode = o->mode;
        h.indel_end_skip = o->indel_end_skip; h.max_del_occ = o->max_del_occ; h.max_entries = o->max_entries;
        h.max_diff = o->max_diff; h.max_gapo = o->max_gapo; h.max_gape = o->max_gape;
        h.max_seed_diff = o->max_seed_diff; h.seed_len = o->seed_len; h.max_top2 = o->max_top2;
        if (o->fnr > 0.0) h.max_diff = galn_cal_maxdiff(bmax[b], 0.02, o->fnr);
        if (h.max_diff < h.max_gapo) h.max_gapo = h.max_diff;
        galn_opts tmp = *o;
        tmp.max_gapo = h.max_gapo;
        h.n_stacks = score_of(h.max_diff + 1, h.max_gapo + 1, h.max_gape + 1, &tmp);
        max_stacks = std::max(max_stacks, h.n_stacks);
        if (h.max_gapo > 126 || h.max_gape > 126) wide = true;
    }
    // bwa_cal_maxdiff by read length: a table per option set with -n as a fraction, over the lengths present
    std::vector<std::vector<int32_t>> md_tab((size_t)n_sets);
    {
        std::vector<uint8_t> seen((size_t)max_len + 1, 0);
        for (const Part &P : parts)
            for (int L = 0; L <= max_len; ++L) seen[(size_t)L] |= P.seen[(size_t)L];
        for (int k = 0; k < n_sets; ++k) {
            if (!(sets[k].fnr > 0.0)) continue;
            int same = -1;   // an earlier set with the same fraction shares its table
            for (int j = 0; j < k && same < 0; ++j)
                if (sets[j].fnr > 0.0 && memcmp(&sets[j].fnr, &sets[k].fnr, 4) == 0) same = j;
            if (same >= 0) { md_tab[(size_t)k] = md_tab[(size_t)same]; continue; }
            md_tab[(size_t)k].assign((size_t)max_len + 1, 0);
            for (int L = 0; L <= max_len; ++L)
                if (seen[(size_t)L]) md_tab[(size_t)k][(size_t)L] = galn_cal_maxdiff(L, 0.02, sets[k].fnr);
        }
    }
    // pass 2: each read's max_diff
    std::vector<uint8_t> wide_t((size_t)T, 0);
    par([&](int r0, int r1, int t) {
        for (int r = r0; r < r1; ++r) {
            const int b = h_bid[r];
            const int k = batch_set ? batch_set[b] : 0;
            const int md = sets[k].fnr > 0.0 ? md_tab[(size_t)k][(size_t)(in->offset[r + 1] - in->offset[r])]
                                             : bopt[(size_t)b].max_diff;
            h_md[r] = md;
            if (md > 125) wide_t[(size_t)t] = 1;
        }
    });
    for (uint8_t w : wide_t) wide = wide || w;
    for (auto &h : bopt) h.wide = wide ? 1 : 0;

    // ---- device buffers ----
    RCK(B.seq.ensure((size_t)std::max<int64_t>(total, 1)));
    RCK(B.query.ensure((size_t)std::max<int64_t>(total, 1)));
    RCK(B.off.ensure((nn + 1) * 8));
    RCK(B.bidx.ensure(nn * 4));
    RCK(B.maxdiff.ensure(nn * 4));
    RCK(B.bopt.ensure(bopt.size() * sizeof(HostBatchOpt)));
    RCK(B.out_n.ensure(nn * 4));
    RCK(B.out_off.ensure(nn * 8));
    RCK(B.out_pops.ensure(nn * 8));
    RCK(B.out_trace.ensure(nn * 8));
    RCK(B.out_peak.ensure(nn * 4));
    RCK(B.out_fetch.ensure(nn * 4));
    RCK(B.out_tier.ensure(nn));
    RCK(B.list_a.ensure(nn * 4));
    RCK(B.list_b.ensure(nn * 4));
    RCK(B.counters.ensure(64));
    RCK(B.rec_top.ensure(64));
    int64_t rec_cap = (int64_t)n * 2 + 65536;
    RCK(B.out_rec.ensure((size_t)rec_cap * 24));
    rec_cap = (int64_t)(B.out_rec.n / 24);
    // reads ordered by batch (stable): each batch is one contiguous segment of the list
    std::vector<int> bstart((size_t)n_batches + 1, 0);
    for (int b = 0; b < n_batches; ++b) bstart[(size_t)b + 1] = bstart[(size_t)b] + bcount[(size_t)b];
    // the fused launch (first tier and warp tier in one launch) for the persistent engine when the warp tier
    // can run: its first tier claims the reads longest expected search first (max_diff, then length), so that
    // heavy reads reach the warp tier early; results do not depend on the order
    // the share of the fused launch's blocks that are warp-tier warps from the start (1 / fused_div; 0: two
    // launches): the autotuner's for this option set, else the index's
    int fused_div = ix->use_fused ? ix->fused_div : 0;
    if (!ix->tune_active) {
        auto it = ix->tuned.find(opts_key(&sets[0]));
        if (it != ix->tuned.end() && it->second.arena > 0) fused_div = it->second.fused_div;
    }
    const bool use_fused = engine == GALN_ENGINE_PERSISTENT && fused_div > 0 && ix->use_warp && !wide && n > 0;
    if (use_fused) {
        const int kL = kWarpMaxLen + 1, nkey = 126 * kL;
        auto key = [&](int r) {
            const int md = std::min(std::max(h_md[r], 0), 125);
            const int len = (int)std::min<int64_t>(in->offset[r + 1] - in->offset[r], kWarpMaxLen);
            return (125 - md) * kL + (kWarpMaxLen - len);   // ascending key = descending (max_diff, length)
        };
        std::vector<int32_t> cnt((size_t)nkey + 1, 0);
        for (int r = 0; r < n; ++r) ++cnt[(size_t)key(r) + 1];
        for (int k = 0; k < nkey; ++k) cnt[(size_t)k + 1] += cnt[(size_t)k];
        for (int r = 0; r < n; ++r) h_list[cnt[(size_t)key(r)]++] = r;
    } else if (sorted) {
        par([&](int r0, int r1, int) { for (int r = r0; r < r1; ++r) h_list[r] = r; });
    } else {
        std::vector<int> fill(bstart.begin(), bstart.end() - 1);
        for (int r = 0; r < n; ++r) h_list[fill[(size_t)bid[r]]++] = r;
    }
    ECK(cudaMemcpyAsync(B.off.p, h_off, (size_t)(n + 1) * 8, cudaMemcpyHostToDevice, st));
    ECK(cudaMemcpyAsync(B.bidx.p, h_bid, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    ECK(cudaMemcpyAsync(B.maxdiff.p, h_md, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    ECK(cudaMemcpyAsync(B.list_a.p, h_list, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    ECK(cudaMemcpyAsync(B.bopt.p, bopt.data(), bopt.size() * sizeof(HostBatchOpt), cudaMemcpyHostToDevice, st));
    ECK(cudaMemsetAsync(B.rec_top.p, 0, 8, st));

    DevJob job;
    job.n_reads = n; job.n_batches = n_batches;
    job.seq = (uint8_t *)B.seq.p; job.query = (uint8_t *)B.query.p; job.off = (int64_t *)B.off.p;
    job.bidx = (int32_t *)B.bidx.p; job.maxdiff = (int32_t *)B.maxdiff.p; job.bopt = (HostBatchOpt *)B.bopt.p;
    job.seed_len = seed_part; job.max_len = max_len; job.max_stacks = max_stacks; job.any_wide = wide ? 1 : 0;
    job.trace = ix->trace ? 1 : 0;
    job.out_n = (int32_t *)B.out_n.p; job.out_off = (int64_t *)B.out_off.p; job.out_pops = (uint64_t *)B.out_pops.p;
    job.out_trace = (uint64_t *)B.out_trace.p; job.out_peak = (int32_t *)B.out_peak.p;
    job.out_fetch = (uint32_t *)B.out_fetch.p; job.out_tier = (int8_t *)B.out_tier.p;
    job.out_rec = (uint64_t *)B.out_rec.p; job.rec_top = (unsigned long long *)B.rec_top.p; job.rec_cap = rec_cap;
    job.list_a = (int32_t *)B.list_a.p; job.list_b = (int32_t *)B.list_b.p; job.counters = (int32_t *)B.counters.p;
    if (job.seed_len < 0) job.seed_len = 0;
    // the occurrence layout: the autotuner's for this option set, else the index's default; the stream's
    // persisting L2 window follows it
    job.occ = ix->occ;
    if (engine != GALN_ENGINE_PLAIN && !ix->tune_active) {
        auto it = ix->tuned.find(opts_key(&sets[0]));
        if (it != ix->tuned.end()) job.occ = it->second.occ;
    }
    if (ctx.l2_occ != job.occ) {
        index_l2_policy(ix, st, job.occ);
        ctx.l2_occ = job.occ;
    }
    cudaEvent_t span0, span1;
    ECK(cudaEventCreate(&span0));
    ECK(cudaEventCreate(&span1));
    ECK(cudaEventRecord(span0, st));
    S.ms_phase[0] = now_ms() - t_start;
    RCK(dev_encode(job, st));
    if (n > 0) S.kernel_launches += 1;
    if (n > 0 && engine != GALN_ENGINE_PLAIN) {
        const int w = index_l2_warm(ix, st, job.occ);
        if (w < 0) return w;
        S.kernel_launches += w;
    }

    size_t free_b = 0, total_b = 0;
    ECK(cudaMemGetInfo(&free_b, &total_b));
    size_t budget = (size_t)((double)(free_b + B.ws.n) * ix->mem_fraction);
    budget = std::min(budget, (size_t)((double)total_b * ix->mem_fraction * ctx.mem_share));

    cudaEvent_t e0, e1;
    ECK(cudaEventCreate(&e0));
    ECK(cudaEventCreate(&e1));
    float k_ms = 0;
    RCK(B.h_misc.ensure(256));   // counters and queue words (16 ints), then the warp counters at byte 128
    int32_t *h_cnt = (int32_t *)B.h_misc.p;

    // run one tier over list[0..m) with overflow going to ovf; returns the overflow count
    auto run_tier = [&](TierCfg cfg, const int32_t *list, int m, int32_t *ovf, int *n_ovf) -> int {
        *n_ovf = 0;
        if (m == 0) return 0;
        if (cfg.persistent) {
            int res = dev_resident_threads(cfg, wide, ix->dev.device);
            if (res <= 0) return GALN_ECUDA;
            cfg.threads = std::min(m, res);
        } else cfg.threads = m;
        if (cfg.threads < 1) cfg.threads = 1;
        // fit the workspace into the budget
        for (;;) {
            size_t need = ws_bytes(cfg, job);
            if (need <= budget || cfg.threads <= cfg.block) break;
            if (!cfg.persistent) return GALN_ENOMEM;   // caller splits
            cfg.threads = std::max(cfg.block, cfg.threads / 2);
        }
        RCK(B.ws.ensure(ws_bytes(cfg, job)));
        S.tier_threads[cfg.tier] = std::max<int64_t>(S.tier_threads[cfg.tier], cfg.threads);
        S.tier_reads[cfg.tier] += m;
        if (cfg.persistent && cfg.tier == 0 && ix->use_graph) {
            // the persistent first-tier launch as a CUDA graph: counter reset, timing events, the kernel and the
            // read-back of the overflow count are captured once and re-instantiated only when the captured
            // graph cannot update the executable one (e.g. a different kernel instantiation)
            cudaGraph_t g = nullptr;
            ECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            cudaMemsetAsync(job.counters, 0, 8, st);
            cudaEventRecordWithFlags(e0, st, cudaEventRecordExternal);   // a timed event node, not a capture join
            int lrc = dev_search(ix->dev, job, cfg, list, m, ovf, B.ws.p, st);
            cudaEventRecordWithFlags(e1, st, cudaEventRecordExternal);
            cudaMemcpyAsync(h_cnt, job.counters, 8, cudaMemcpyDeviceToHost, st);
            cudaError_t ce = cudaStreamEndCapture(st, &g);
            if (lrc || ce != cudaSuccess) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return lrc ? lrc : GALN_ECUDA; }
            bool updated = false;
            if (ctx.graph_exec) {
                cudaGraphExecUpdateResultInfo info;
                updated = cudaGraphExecUpdate(ctx.graph_exec, g, &info) == cudaSuccess;
                if (!updated) { cudaGetLastError(); cudaGraphExecDestroy(ctx.graph_exec); ctx.graph_exec = nullptr; }
            }
            if (!updated) {
                cudaError_t ie = cudaGraphInstantiate(&ctx.graph_exec, g, 0);
                if (ie != cudaSuccess) { cudaGraphDestroy(g); ctx.graph_exec = nullptr; return GALN_ECUDA; }
            }
            cudaGraphDestroy(g);
            S.ms_phase[5] = now_ms() - t_start;
            ECK(cudaGraphLaunch(ctx.graph_exec, st));
            ECK(cudaStreamSynchronize(st));
            S.graph_launches += 1;
        } else {
            ECK(cudaMemsetAsync(job.counters, 0, 8, st));
            ECK(cudaEventRecord(e0, st));
            RCK(dev_search(ix->dev, job, cfg, list, m, ovf, B.ws.p, st));
            ECK(cudaEventRecord(e1, st));
            ECK(cudaMemcpyAsync(h_cnt, job.counters, 8, cudaMemcpyDeviceToHost, st));
            ECK(cudaStreamSynchronize(st));
        }
        float ms = 0;
        ECK(cudaEventElapsedTime(&ms, e0, e1));
        k_ms += ms;
        S.ms_tier[cfg.tier] += ms;
        S.kernel_launches += 1;
        *n_ovf = h_cnt[1];
        return 0;
    };

    // ---- T0 ----
    int32_t *cur = job.list_a, *nxt = job.list_b;
    int n_ovf = 0;
    TierCfg t0;
    t0.tier = 0;
    t0.freelist = false; t0.aln_cap = ix->t0_aln; t0.block = ix->t0_block;
    t0.cap = engine == GALN_ENGINE_PLAIN ? ix->plain_t0_cap : ix->t0_cap;
    if (engine != GALN_ENGINE_PLAIN && !ix->tune_active && !ix->tuned.empty()) {
        // the autotuner's choice for this option set (single-set jobs; mixed jobs use the first set's)
        auto it = ix->tuned.find(opts_key(&sets[0]));
        if (it != ix->tuned.end()) { t0.cap = it->second.cap; t0.block = it->second.block; }
    }
    // the warp tier's arena per warp and its big-arena warps: the autotuner's for this option set, else the
    // index's
    int arena = ix->warp_arena, n_big_max = ix->warp_big;
    if (!ix->tune_active) {
        auto it = ix->tuned.find(opts_key(&sets[0]));
        if (it != ix->tuned.end() && it->second.arena > 0) { arena = it->second.arena; n_big_max = it->second.big; }
    }
    // the cut-off, one wave's staged pushes and a partly filled chunk per bucket
    const int64_t full_chunks = (max_entries_all + 16 + 3 * 32 * 128 + kWarpMaxStacks * kWarpChunk) / kWarpChunk
                                + kWarpMaxStacks + 1;
    const int big_chunks = (int)std::min<int64_t>(std::max<int64_t>(full_chunks, arena), 1 << 22);
    const int aln_cap_w = 4096;
    const bool warp_ok = ix->use_warp && !wide && engine != GALN_ENGINE_PLAIN;
    unsigned long long *h_dbg = (unsigned long long *)((char *)B.h_misc.p + 128);
    bool fused = false;
    std::vector<int32_t> elig, rest;     // reads for the warp tier's next pass, and for the thread tiers
    if (use_fused) {
        // one persistent launch of both tiers: blocks of kFusedWarps warps, as many as stay resident; 1 / fused_div
        // of them are warp-tier warps from the start, the others run the first tier first
        const int grid = fused_resident_blocks(ix->dev.device);
        if (grid <= 1) return GALN_ECUDA;
        const int n_w_blocks = std::min(grid - 1, std::max(1, grid / fused_div));
        TierCfg ft = t0;
        ft.persistent = true;
        ft.threads = (grid - n_w_blocks) * kFusedWarps * 32;
        ft.block = kFusedWarps * 32;
        WarpCfg wc;
        wc.n_warps = grid * kFusedWarps;
        wc.aln_cap = aln_cap_w;
        wc.arena_chunks = arena;
        wc.big_chunks = big_chunks;
        wc.q_wait_ns = ix->warp_wait_ns;
        wc.n_big = big_chunks > arena ? std::min(n_big_max, n_w_blocks * kFusedWarps) : 0;
        while (wc.n_big > 0 && fused_ws_bytes(ft, job, wc, n) > budget) wc.n_big /= 2;
        while (wc.arena_chunks > 1024 && fused_ws_bytes(ft, job, wc, n) > budget) wc.arena_chunks /= 2;
        if (fused_ws_bytes(ft, job, wc, n) <= budget) {
            RCK(B.ws.ensure(fused_ws_bytes(ft, job, wc, n)));
            unsigned long long *dbg = nullptr;
            if (ix->keep_stats) {
                RCK(B.dbg.ensure(kWarpDbg * 8));
                dbg = (unsigned long long *)B.dbg.p;
            }
            FusedQueues fq;
            fused_queues(ft, job, wc, n, B.ws.p, fq);
            // counters, timing events, the launch and the read-back of its counters and queue control words,
            // captured once as a CUDA graph and updated in place when only parameters change
            auto record = [&]() -> int {
                if (cudaMemsetAsync(job.counters, 0, 64, st) != cudaSuccess) return GALN_ECUDA;
                if (dbg && cudaMemsetAsync(dbg, 0, kWarpDbg * 8, st) != cudaSuccess) return GALN_ECUDA;
                if (cudaEventRecordWithFlags(e0, st, cudaEventRecordExternal) != cudaSuccess) return GALN_ECUDA;
                int lrc = dev_search_fused(ix->dev, job, ft, wc, n_w_blocks, cur, n, nxt, B.ws.p, st, dbg);
                if (lrc) return lrc;
                if (cudaEventRecordWithFlags(e1, st, cudaEventRecordExternal) != cudaSuccess) return GALN_ECUDA;
                if (cudaMemcpyAsync(h_cnt, job.counters, 16, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaMemcpyAsync(h_cnt + 4, fq.hq_ctl, 16, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaMemcpyAsync(h_cnt + 8, fq.q_ctl, 16, cudaMemcpyDeviceToHost, st) != cudaSuccess)
                    return GALN_ECUDA;
                if (dbg && cudaMemcpyAsync(h_dbg, dbg, kWarpDbg * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess)
                    return GALN_ECUDA;
                return 0;
            };
            if (ix->use_graph) {
                cudaGraph_t g = nullptr;
                ECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                const int lrc = record();
                cudaError_t ce = cudaStreamEndCapture(st, &g);
                if (lrc || ce != cudaSuccess) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return lrc ? lrc : GALN_ECUDA; }
                bool updated = false;
                if (ctx.fused_exec) {
                    cudaGraphExecUpdateResultInfo info;
                    updated = cudaGraphExecUpdate(ctx.fused_exec, g, &info) == cudaSuccess;
                    if (!updated) { cudaGetLastError(); cudaGraphExecDestroy(ctx.fused_exec); ctx.fused_exec = nullptr; }
                }
                if (!updated && cudaGraphInstantiate(&ctx.fused_exec, g, 0) != cudaSuccess) {
                    cudaGraphDestroy(g);
                    ctx.fused_exec = nullptr;
                    return GALN_ECUDA;
                }
                cudaGraphDestroy(g);
                ECK(cudaGraphLaunch(ctx.fused_exec, st));
                S.graph_launches += 1;
            } else {
                RCK(record());
            }
            ECK(cudaStreamSynchronize(st));
            float ms = 0;
            ECK(cudaEventElapsedTime(&ms, e0, e1));
            k_ms += ms;
            S.ms_tier[0] += ms;
            S.kernel_launches += 1;
            S.fused = true;
            S.tier_threads[0] = ft.threads;
            S.tier_threads[1] = (int64_t)wc.n_warps * 32;
            S.tier_reads[0] += n;
            if (dbg)
                for (int q = 0; q < kWarpDbg; ++q) S.warp_dbg[q] = h_dbg[q];
            // what the launch left: the first tier's overflow the warp tier cannot take, the warp tier's
            // overflow, and reads still queued (all that were ever queued when a slot was lost)
            const int t0_ovf = h_cnt[1], w_ovf = h_cnt[3];
            const int hq_head = h_cnt[4], hq_tail = h_cnt[5], hq_lost = h_cnt[7];
            const int bq_head = h_cnt[8], bq_tail = h_cnt[9], bq_lost = h_cnt[11];
            S.overflow_reads[0] = t0_ovf;
            S.tier_reads[1] += hq_tail;
            S.warp_queued = (int64_t)bq_tail + hq_tail;
            S.warp_gave_up = (hq_lost || bq_lost) ? 1 : 0;
            const int hq_from = hq_lost ? 0 : std::min(hq_head, hq_tail);
            const int bq_from = bq_lost ? 0 : std::min(bq_head, bq_tail);
            const int n_hq = std::max(0, hq_tail - hq_from), n_bq = wc.n_big > 0 ? std::max(0, bq_tail - bq_from) : 0;
            rest.resize((size_t)t0_ovf);
            elig.resize((size_t)w_ovf + n_hq + n_bq);
            if (t0_ovf) ECK(cudaMemcpyAsync(rest.data(), nxt, (size_t)t0_ovf * 4, cudaMemcpyDeviceToHost, st));
            if (w_ovf) ECK(cudaMemcpyAsync(elig.data(), fq.w_ovf, (size_t)w_ovf * 4, cudaMemcpyDeviceToHost, st));
            if (n_hq) ECK(cudaMemcpyAsync(elig.data() + w_ovf, fq.hq + hq_from, (size_t)n_hq * 4, cudaMemcpyDeviceToHost, st));
            if (n_bq)
                ECK(cudaMemcpyAsync(elig.data() + w_ovf + n_hq, fq.big_slots + bq_from, (size_t)n_bq * 4,
                                    cudaMemcpyDeviceToHost, st));
            ECK(cudaStreamSynchronize(st));
            for (int32_t r : rest)
                if (r < 0 || r >= n) return GALN_ECUDA;
            for (int32_t r : elig)
                if (r < 0 || r >= n) return GALN_ECUDA;   // a slot written by no warp
            if (hq_lost || bq_lost) {   // a read may be both queued and in an overflow list
                std::sort(elig.begin(), elig.end());
                elig.erase(std::unique(elig.begin(), elig.end()), elig.end());
            }
            fused = true;
        }
    }
    if (fused) {
        // the warp tier's second pass and the thread tiers follow
    } else if (engine == GALN_ENGINE_PERSISTENT) {
        t0.persistent = true;
        RCK(run_tier(t0, cur, n, nxt, &n_ovf));
        S.ms_phase[3] = now_ms() - t_start;
    } else {
        // one launch per bwa batch, one thread per read; a batch too large for the memory budget is
        // launched in equal chunks
        t0.persistent = false;
        int max_chunk = kBatchReads;
        for (;;) {
            TierCfg probe = t0;
            probe.threads = max_chunk;
            if (ws_bytes(probe, job) <= budget || max_chunk <= 1024) break;
            max_chunk /= 2;
        }
        int acc = 0;
        for (int b = 0; b < n_batches; ++b) {
            for (int s0 = bstart[b]; s0 < bstart[b + 1]; s0 += max_chunk) {
                int m = std::min(max_chunk, bstart[b + 1] - s0);
                int got = 0;
                RCK(run_tier(t0, cur + s0, m, nxt + acc, &got));
                acc += got;
            }
        }
        n_ovf = acc;
    }
    if (!fused) S.overflow_reads[0] = n_ovf;
    std::swap(cur, nxt);

    // ---- W: the warp tier for the reads that overflowed T0 (those it can take); after the fused launch,
    // its second pass for what that launch left ----
    if (warp_ok && (fused || n_ovf > 0)) {
        // longest expected searches first, so that the heaviest reads do not start last and run alone at the
        // end of the launch; results do not depend on the order. Order 1: the reads whose first-tier search
        // overflowed after the fewest pops (the stack grew fastest) first, read from the first tier's pop
        // counts; order 0: max_diff, then length. Counting sorts: the eligible reads have max_diff <= 125 and
        // length <= kWarpMaxLen; pop counts are clamped.
        const int kL = kWarpMaxLen + 1, nkey = 126 * kL;
        auto warp_key = [&](int32_t r) {
            const int md = std::min(std::max(maxdiff[r], 0), 125);
            const int len = (int)(in->offset[r + 1] - in->offset[r]);
            return (125 - md) * kL + (kWarpMaxLen - len);   // ascending key = descending (max_diff, length)
        };
        bool elig_sorted = false;
        if (!fused) {
            // The overflow list into pinned memory (the read list's host copy went to the device at the start),
            // then, on the host threads, each read's eligibility and key, per-thread key counts, and a stable
            // scatter: the device waits for this gap, so it is kept to a few passes over pinned arrays.
            ECK(cudaMemcpyAsync(h_list, cur, (size_t)n_ovf * 4, cudaMemcpyDeviceToHost, st));
            ECK(cudaStreamSynchronize(st));
            const int TT = n_ovf >= (1 << 15) ? T : 1;
            const bool by_key = ix->warp_order != 1;
            std::vector<std::vector<int32_t>> cnt_t((size_t)TT);
            std::vector<int64_t> n_el((size_t)TT, 0), n_rest((size_t)TT, 0);
            auto chunk = [&](int t) { return std::make_pair((int)((int64_t)n_ovf * t / TT), (int)((int64_t)n_ovf * (t + 1) / TT)); };
            auto eligible = [&](int32_t r) {
                const int len = (int)(in->offset[r + 1] - in->offset[r]);
                const HostBatchOpt &h = bopt[bid[r]];
                return len <= kWarpMaxLen && h.n_stacks <= kWarpMaxStacks && h.n_stacks > 0 && h.s_mm > 0 &&
                       h.s_gapo > 0 && h.s_gape > 0;
            };
            auto run_t = [&](const std::function<void(int)> &fn) {
                if (TT == 1) { fn(0); return; }
                std::vector<std::thread> th;
                for (int t = 0; t < TT; ++t) th.emplace_back(fn, t);
                for (auto &x : th) x.join();
            };
            run_t([&](int t) {
                std::vector<int32_t> &c = cnt_t[(size_t)t];
                if (by_key) c.assign((size_t)nkey, 0);
                const auto [i0, i1] = chunk(t);
                for (int i = i0; i < i1; ++i) {
                    const int32_t r = h_list[i];
                    if (r < 0 || r >= n) { n_rest[(size_t)t] = -1; return; }   // a slot written by no thread
                    if (!eligible(r)) { ++n_rest[(size_t)t]; continue; }
                    ++n_el[(size_t)t];
                    if (by_key) ++c[(size_t)warp_key(r)];
                }
            });
            for (int t = 0; t < TT; ++t) if (n_rest[(size_t)t] < 0) return GALN_ECUDA;
            // where each thread's reads of each key go: keys ascending, threads in order within a key
            std::vector<int64_t> el0((size_t)TT + 1, 0), rs0((size_t)TT + 1, 0);
            for (int t = 0; t < TT; ++t) { el0[(size_t)t + 1] = el0[(size_t)t] + n_el[(size_t)t]; rs0[(size_t)t + 1] = rs0[(size_t)t] + n_rest[(size_t)t]; }
            if (by_key) {
                int32_t run = 0;
                for (int k = 0; k < nkey; ++k)
                    for (int t = 0; t < TT; ++t) {
                        const int32_t v = cnt_t[(size_t)t][(size_t)k];
                        cnt_t[(size_t)t][(size_t)k] = run;
                        run += v;
                    }
            }
            rest.resize((size_t)rs0[(size_t)TT]);
            run_t([&](int t) {
                std::vector<int32_t> &c = cnt_t[(size_t)t];
                int64_t e = el0[(size_t)t], q = rs0[(size_t)t];
                const auto [i0, i1] = chunk(t);
                for (int i = i0; i < i1; ++i) {
                    const int32_t r = h_list[i];
                    if (!eligible(r)) rest[(size_t)q++] = r;
                    else if (by_key) h_wlist[c[(size_t)warp_key(r)]++] = r;
                    else h_wlist[e++] = r;
                }
            });
            elig.assign(h_wlist, h_wlist + el0[(size_t)TT]);
            elig_sorted = by_key;
        }
        if (!fused && ix->warp_order == 1 && !elig.empty()) {
            RCK(B.h_pops.ensure((size_t)n * 8));
            uint64_t *hp = (uint64_t *)B.h_pops.p;
            ECK(cudaMemcpyAsync(hp, job.out_pops, (size_t)n * 8, cudaMemcpyDeviceToHost, st));
            ECK(cudaStreamSynchronize(st));
            const int kMaxKey = 1 << 16;
            std::vector<int32_t> cnt((size_t)kMaxKey + 1, 0), sorted(elig.size());
            auto key = [&](int32_t r) { return (int)std::min<uint64_t>(hp[r], (uint64_t)kMaxKey - 1); };
            for (int32_t r : elig) ++cnt[(size_t)key(r) + 1];
            for (int k = 0; k < kMaxKey; ++k) cnt[(size_t)k + 1] += cnt[(size_t)k];
            for (int32_t r : elig) sorted[(size_t)cnt[(size_t)key(r)]++] = r;
            elig.swap(sorted);
        } else if (!elig_sorted) {
            std::vector<int32_t> cnt((size_t)nkey + 1, 0), sorted(elig.size());
            for (int32_t r : elig) ++cnt[(size_t)warp_key(r) + 1];
            for (int k = 0; k < nkey; ++k) cnt[(size_t)k + 1] += cnt[(size_t)k];
            for (int32_t r : elig) sorted[(size_t)cnt[(size_t)warp_key(r)]++] = r;
            elig.swap(sorted);
        }
        // pass 1: the tuned arena per warp, plus up to n_big_max warps whose arenas hold the max_entries
        // cut-off and take over, in the same launch, the reads that outgrow the small ones (the fused launch
        // is this pass); pass 2, only for reads still queued or not finished when pass 1 ended, with big
        // arenas for every warp
        for (int pass = fused ? 1 : 0; pass < 2 && !elig.empty(); ++pass) {
            int ne = (int)elig.size();
            int res_w = warp_resident(ix->dev.device);
            if (res_w <= 0) return GALN_ECUDA;
            WarpCfg wc;
            wc.aln_cap = aln_cap_w;
            wc.n_warps = std::min(ne, res_w);
            wc.arena_chunks = arena;
            wc.big_chunks = big_chunks;
            wc.q_wait_ns = ix->warp_wait_ns;
            if (pass == 0) {
                wc.n_big = std::min(n_big_max, wc.n_warps / 8);
                if (big_chunks <= wc.arena_chunks) wc.n_big = 0;
                while (wc.n_big > 0 && warp_ws_bytes(wc, ne) > budget) wc.n_big /= 2;
                while (wc.arena_chunks > 1024 && warp_ws_bytes(wc, ne) > budget) wc.arena_chunks /= 2;
                while (wc.n_warps > 1 && warp_ws_bytes(wc, ne) > budget) {
                    wc.n_warps /= 2;
                    wc.n_big = std::min(wc.n_big, wc.n_warps / 8);
                }
            } else {
                wc.n_warps = std::min(wc.n_warps, 256);   // few reads get here; keep the big arenas' footprint bounded
                wc.arena_chunks = big_chunks;
                wc.n_big = 0;
                while (wc.n_warps > 1 && warp_ws_bytes(wc, ne) > budget) wc.n_warps /= 2;
            }
            RCK(B.ws.ensure(warp_ws_bytes(wc, ne)));
            // the first pass's list from its pinned copy
            ECK(cudaMemcpyAsync(cur, pass == 0 && elig_sorted ? h_wlist : elig.data(), (size_t)ne * 4,
                                cudaMemcpyHostToDevice, st));
            ECK(cudaMemsetAsync(job.counters, 0, 8, st));
            unsigned long long *dbg = nullptr;
            if (ix->keep_stats) {
                RCK(B.dbg.ensure(kWarpDbg * 8));
                dbg = (unsigned long long *)B.dbg.p;
                ECK(cudaMemsetAsync(dbg, 0, kWarpDbg * 8, st));
            }
            ECK(cudaEventRecord(e0, st));
            if (pass == 0) S.ms_phase[4] = now_ms() - t_start;
            RCK(dev_search_warp(ix->dev, job, wc, 1, cur, ne, nxt, B.ws.p, st, dbg));
            ECK(cudaEventRecord(e1, st));
            int32_t *q_slots = nullptr;
            int32_t *q_ctl = warp_queue(wc, ne, B.ws.p, &q_slots);
            ECK(cudaMemcpyAsync(h_cnt, job.counters, 8, cudaMemcpyDeviceToHost, st));
            ECK(cudaMemcpyAsync(h_cnt + 4, q_ctl, 16, cudaMemcpyDeviceToHost, st));
            if (dbg) {
                unsigned long long hd[kWarpDbg];
                ECK(cudaMemcpyAsync(hd, dbg, sizeof(hd), cudaMemcpyDeviceToHost, st));
                ECK(cudaStreamSynchronize(st));
                for (int q = 0; q < kWarpDbg; ++q)
                    S.warp_dbg[q] = q == kWarpDbg - 1 ? std::max<uint64_t>(S.warp_dbg[q], hd[q]) : S.warp_dbg[q] + hd[q];
            }
            ECK(cudaStreamSynchronize(st));
            float ms = 0;
            ECK(cudaEventElapsedTime(&ms, e0, e1));
            k_ms += ms;
            S.ms_tier[1] += ms;
            S.tier_threads[1] = std::max<int64_t>(S.tier_threads[1], (int64_t)wc.n_warps * 32);
            S.tier_reads[1] += ne;
            S.kernel_launches += 1;
            // the reads pass 1 could not finish: its overflow list, then the reads still queued for a big
            // warp (all queued reads if a queue slot was lost)
            const int got = h_cnt[1];
            const int q_head = h_cnt[4], q_tail = h_cnt[5], q_lost = h_cnt[7];
            const int q_from = q_lost ? 0 : std::min(q_head, q_tail);
            const int n_q = wc.n_big > 0 ? std::max(0, q_tail - q_from) : 0;
            std::vector<int32_t> wov((size_t)got + n_q);
            if (got) ECK(cudaMemcpyAsync(wov.data(), nxt, (size_t)got * 4, cudaMemcpyDeviceToHost, st));
            if (n_q) ECK(cudaMemcpyAsync(wov.data() + got, q_slots + q_from, (size_t)n_q * 4, cudaMemcpyDeviceToHost, st));
            if (got || n_q) ECK(cudaStreamSynchronize(st));
            for (int32_t r : wov)
                if (r < 0 || r >= n) return GALN_ECUDA;   // a slot written by no warp
            if (q_lost) {   // every queued read again: one may also be in the overflow list
                std::sort(wov.begin(), wov.end());
                wov.erase(std::unique(wov.begin(), wov.end()), wov.end());
            }
            if (pass == 0) { S.warp_queued = q_tail; S.warp_gave_up = q_lost ? 1 : 0; }
            if (pass == 1) S.overflow_reads[1] = (int64_t)wov.size();
            elig.swap(wov);
        }
        rest.insert(rest.end(), elig.begin(), elig.end());
        n_ovf = (int)rest.size();
        if (n_ovf) {
            ECK(cudaMemcpyAsync(cur, rest.data(), (size_t)n_ovf * 4, cudaMemcpyHostToDevice, st));
            ECK(cudaStreamSynchronize(st));
        }
    }

    // ---- T1, T2, ... (tiers 2..7 in the statistics) ----
    int tier = 2;
    int64_t aln_cap = ix->t1_aln;
    while (n_ovf > 0 && tier < 8) {
        // make room for records: grow the record buffer when it is more than half used
        unsigned long long top = 0;
        ECK(cudaMemcpyAsync(&top, job.rec_top, 8, cudaMemcpyDeviceToHost, st));
        ECK(cudaStreamSynchronize(st));
        if ((int64_t)top > job.rec_cap / 2) {
            int64_t keep = std::min<int64_t>((int64_t)top, job.rec_cap);
            int64_t cap2 = std::max<int64_t>(2 * job.rec_cap, (int64_t)top * 2 + 65536);
            void *np = nullptr;
            ECK(cudaMalloc(&np, (size_t)cap2 * 24));
            ECK(cudaMemcpyAsync(np, job.out_rec, (size_t)keep * 24, cudaMemcpyDeviceToDevice, st));
            ECK(cudaStreamSynchronize(st));
            B.out_rec.release();
            B.out_rec.p = np;
            B.out_rec.n = (size_t)cap2 * 24;
            job.out_rec = (uint64_t *)np;
            job.rec_cap = cap2;
            if ((int64_t)top > job.rec_cap) ECK(cudaMemcpyAsync(job.rec_top, &keep, 8, cudaMemcpyHostToDevice, st));
        }
        TierCfg t;
        t.tier = tier;
        t.freelist = true;
        t.persistent = true;
        t.block = 128;
        // live entries: t1_cap, then 2^19, then enough for the max_entries cut-off
        int64_t full = std::min<int64_t>(max_entries_all + 16, 0x7fffffff);
        t.cap = tier == 2 ? ix->t1_cap : tier == 3 ? (int)std::min<int64_t>(full, 1 << 19) : (int)full;
        if (t.cap < 16) t.cap = 16;
        t.aln_cap = (int)std::min<int64_t>(aln_cap, 1 << 24);
        int got = 0;
        RCK(run_tier(t, cur, n_ovf, nxt, &got));
        S.overflow_reads[tier] = got;
        n_ovf = got;
        std::swap(cur, nxt);
        if (tier >= 3) aln_cap *= 16;
        else aln_cap = 65536;
        ++tier;
    }
    S.tiers = tier;
    ECK(cudaEventRecord(span1, st));
    ECK(cudaEventSynchronize(span1));
    {
        float ms = 0;
        ECK(cudaEventElapsedTime(&ms, span0, span1));
        S.ms_device = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(span0);
    cudaEventDestroy(span1);
    if (n_ovf > 0) return GALN_ENOMEM;

    // ---- results: put in read order on the device, then one copy of each array into the caller's results ----
    S.ms_phase[1] = now_ms() - t_start;
    RCK(B.rec_off.ensure((nn + 1) * 8));
    RCK(B.rec_ord.ensure((size_t)std::max<int64_t>(job.rec_cap, 1) * 24));
    RCK(B.tile.ensure(order_tile_bytes(n)));
    RCK(dev_order_results(job, n, (int64_t *)B.rec_off.p, (uint64_t *)B.rec_ord.p, (int64_t *)B.tile.p, st));
    int64_t *h_total = (int64_t *)B.h_misc.p + 4;
    *h_total = 0;
    if (n > 0) ECK(cudaMemcpyAsync(h_total, (int64_t *)B.rec_off.p + n, 8, cudaMemcpyDeviceToHost, st));
    ECK(cudaStreamSynchronize(st));
    const int64_t n_rec = *h_total;
    if (n_rec < 0 || n_rec > job.rec_cap) return GALN_ECUDA;
    auto *P = new ResultsPriv();
    P->n_aln.resize(nn);
    P->rec_off.resize(nn + 1);
    P->rec.resize((size_t)std::max<int64_t>(n_rec, 1));
    P->pops.resize(nn);
    P->trace.resize(nn);
    P->rec_off[0] = 0;
    cudaError_t ce = cudaSuccess;
    if (n > 0) {
        // one copy into reused pinned memory, then the result arrays filled by several host threads
        const size_t b_n = (size_t)n * 4, b_off = ((size_t)n + 1) * 8, b_rec = (size_t)n_rec * 24, b_p = (size_t)n * 8;
        const size_t o_off = (b_n + 255) & ~(size_t)255, o_rec = o_off + ((b_off + 255) & ~(size_t)255);
        const size_t o_pops = o_rec + ((b_rec + 255) & ~(size_t)255), o_trace = o_pops + ((b_p + 255) & ~(size_t)255);
        if (B.h_res.ensure(o_trace + b_p)) { delete P; return GALN_ENOMEM; }
        char *hr = (char *)B.h_res.p;
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(hr, job.out_n, b_n, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(hr + o_off, B.rec_off.p, b_off, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess && n_rec) ce = cudaMemcpyAsync(hr + o_rec, B.rec_ord.p, b_rec, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(hr + o_pops, job.out_pops, b_p, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(hr + o_trace, job.out_trace, b_p, cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess && ix->keep_stats) {
            S.fetch.resize(nn);
            S.tier_of.resize(nn);
            ce = cudaMemcpyAsync(S.fetch.data(), job.out_fetch, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(S.tier_of.data(), job.out_tier, (size_t)n, cudaMemcpyDeviceToHost, st);
        }
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
        if (ce == cudaSuccess) {
            struct Piece { void *dst; const char *src; size_t bytes; };
            const Piece pieces[5] = {{P->n_aln.data(), hr, b_n}, {P->rec_off.data(), hr + o_off, b_off},
                                     {P->rec.data(), hr + o_rec, b_rec}, {P->pops.data(), hr + o_pops, b_p},
                                     {P->trace.data(), hr + o_trace, b_p}};
            const size_t all = b_n + b_off + b_rec + 2 * b_p;
            const int TT = all >= ((size_t)16 << 20) ? (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency())) : 1;
            auto copy_part = [&](int t) {   // thread t copies its share of every array
                for (const Piece &pc : pieces) {
                    const size_t c0 = pc.bytes * (size_t)t / (size_t)TT, c1 = pc.bytes * (size_t)(t + 1) / (size_t)TT;
                    if (c1 > c0) memcpy((char *)pc.dst + c0, pc.src + c0, c1 - c0);
                }
            };
            if (TT == 1) copy_part(0);
            else {
                std::vector<std::thread> th;
                for (int t = 0; t < TT; ++t) th.emplace_back(copy_part, t);
                for (auto &x : th) x.join();
            }
        }
    }
    if (ce != cudaSuccess) {
        delete P;
        fprintf(stderr, "[galn] CUDA error %s copying results\n", cudaGetErrorString(ce));
        return GALN_ECUDA;
    }
    P->publish(out, n);
    S.ms_phase[2] = now_ms() - t_start;
    S.ms_kernels = k_ms;
    S.ms_total = now_ms() - t_start;
    return 0;
}

}  // namespace galn

extern "C" int galn_aln_run_batch(galn_index *ix, const galn_opts *o, const galn_reads *in, int engine, galn_results *out)
{
    if (!ix || !o || !in || !out) return GALN_EINVAL;
    if (engine != GALN_ENGINE_PLAIN && engine != GALN_ENGINE_PERSISTENT) return GALN_EINVAL;
    memset(out, 0, sizeof(*out));
    std::lock_guard<std::mutex> lk(ix->mu);
    return galn::run_job(ix, ix->main, o, in, engine, out);
}

extern "C" int galn_last_run_stats(galn_index *ix, double *ms_total, double *ms_kernels, int *tiers,
                                   int64_t *launches, int64_t *overflow /* 8 */)
{
    if (!ix) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    if (ms_total) *ms_total = ix->main.last.ms_total;
    if (ms_kernels) *ms_kernels = ix->main.last.ms_kernels;
    if (tiers) *tiers = ix->main.last.tiers;
    if (launches) *launches = ix->main.last.kernel_launches;
    if (overflow) memcpy(overflow, ix->main.last.overflow_reads, sizeof(ix->main.last.overflow_reads));
    return 0;
}

extern "C" int galn_last_run_profile(galn_index *ix, double *ms_device, double *ms_tier, int64_t *tier_reads,
                                     int64_t *tier_threads, uint32_t *fetch, int8_t *tier, int32_t n)
{
    if (!ix) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    if (ms_device) *ms_device = ix->main.last.ms_device;
    if (ms_tier) memcpy(ms_tier, ix->main.last.ms_tier, sizeof(ix->main.last.ms_tier));
    if (tier_reads) memcpy(tier_reads, ix->main.last.tier_reads, sizeof(ix->main.last.tier_reads));
    if (tier_threads) memcpy(tier_threads, ix->main.last.tier_threads, sizeof(ix->main.last.tier_threads));
    if (fetch || tier) {
        if ((size_t)n > ix->main.last.fetch.size()) return GALN_EINVAL;
        if (fetch) memcpy(fetch, ix->main.last.fetch.data(), (size_t)n * 4);
        if (tier) memcpy(tier, ix->main.last.tier_of.data(), (size_t)n);
    }
    return 0;
}

extern "C" int galn_last_graph_launches(galn_index *ix, int64_t *graph_launches)
{
    if (!ix || !graph_launches) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    *graph_launches = ix->main.last.graph_launches;
    return 0;
}

extern "C" int galn_last_run_phases(galn_index *ix, double *ms, int n)
{
    if (!ix || !ms || n < 0) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    const galn::RunStats &S = ix->main.last;
    const double v[8] = {S.ms_phase[0], S.ms_phase[1], S.ms_phase[2], S.ms_total, S.ms_device, S.ms_phase[3],
                         S.ms_phase[4], S.ms_phase[5]};
    for (int q = 0; q < n && q < 8; ++q) ms[q] = v[q];
    return 0;
}

extern "C" int galn_last_warp_counters(galn_index *ix, uint64_t *counters, int n)
{
    if (!ix || !counters || n < 1) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    for (int q = 0; q < n && q < galn::kWarpDbg; ++q) counters[q] = ix->main.last.warp_dbg[q];
    return 0;
}

extern "C" int galn_index_set_l2_persist(galn_index *ix, int on)
{
    if (!ix) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    ix->l2_persist = on != 0;
    if (ix->l2_persist) galn::index_l2_policy(ix, ix->stream, ix->main.l2_occ ? ix->main.l2_occ : ix->occ);
    else galn::index_l2_clear(ix, ix->stream);
    return 0;
}

extern "C" int galn_index_set_occ_layout(galn_index *ix, int stride)
{
    if (!ix || (stride != 64 && stride != 80)) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    ix->occ = stride;
    return 0;
}

extern "C" int galn_index_set_warp_tier(galn_index *ix, int on, int arena_chunks)
{
    if (!ix || arena_chunks < 32) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    ix->use_warp = on != 0;
    ix->warp_arena = arena_chunks;
    return 0;
}

extern "C" int galn_index_set_warp_order(galn_index *ix, int order)
{
    if (!ix || order < 0 || order > 1) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    ix->warp_order = order;
    return 0;
}

extern "C" int galn_index_set_fused(galn_index *ix, int on)
{
    if (!ix) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    ix->use_fused = on != 0;
    return 0;
}

extern "C" int galn_last_run_fused(galn_index *ix, int *fused)
{
    if (!ix || !fused) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    *fused = ix->main.last.fused ? 1 : 0;
    return 0;
}

extern "C" int galn_index_set_warp_wait(galn_index *ix, int64_t wait_ns)
{
    if (!ix || wait_ns < 0) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    ix->warp_wait_ns = (uint64_t)wait_ns;
    return 0;
}

extern "C" int galn_last_warp_queue(galn_index *ix, int64_t *queued, int *gave_up)
{
    if (!ix) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    if (queued) *queued = ix->main.last.warp_queued;
    if (gave_up) *gave_up = ix->main.last.warp_gave_up;
    return 0;
}

extern "C" int galn_index_set_trace(galn_index *ix, int on)
{
    if (!ix) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    ix->trace = on != 0;
    return 0;
}

extern "C" int galn_index_set_tuning(galn_index *ix, int t0_cap, int t0_aln, int t0_block, int t1_cap, int t1_aln,
                                     int keep_stats)
{
    if (!ix) return GALN_EINVAL;
    if (t0_cap < 16 || t0_aln < 1 || t1_cap < 16 || t1_aln < 1 || (t0_block != 64 && t0_block != 128 &&
        t0_block != 256 && t0_block != 512)) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    ix->t0_cap = t0_cap; ix->t0_aln = t0_aln; ix->t0_block = t0_block;
    ix->t1_cap = t1_cap; ix->t1_aln = t1_aln;
    ix->keep_stats = keep_stats != 0;
    return 0;
}
