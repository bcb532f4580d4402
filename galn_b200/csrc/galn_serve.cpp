// galn_serve.cpp -- continuous batching of alignment requests on a resident index.
//
// Requests (each with its own options and its own bwa batch boundaries) are copied in by galn_aln_submit.
// A scheduler thread runs steps back to back. Each step takes up to `step_reads` reads from the admitted
// requests -- every request first gets an equal share, what is left goes to the oldest -- and searches them
// together in one pass of the device tiers, so requests share the same kernels. A request that arrives
// while a step runs joins the next step; a request leaves as soon as its last read has been searched.
// Admission is by the device memory the requests' search stacks need (the reference sizes its warps and
// stack arenas from free device memory, src/galn.cu:908-965): each request's need comes from its option set
// and size (request_stack_need: a first-tier stack per read in flight, sized by n_stacks and the longest read,
// and the max_entries-deep arenas of the heavy-read warps its reads can occupy), and a queued request is
// admitted only while the needs of the admitted requests fit the server's stack budget. A request that does
// not fit waits while later, smaller ones are admitted past it, up to kMaxBypass of them; then admission
// waits until it fits (it is admitted alone at worst, so nothing waits for ever). max_active bounds the
// requests in flight as well. Several steps run at once (n_workers, each with its own stream and device
// buffers), so the last heavy reads of one step overlap the next step's work on the device.
//
// Results do not depend on what else is in a step: each read's options are its request's, and each bwa
// batch's options come from the longest read of that batch in its own request (batch_max_len), whether the
// request is searched in one step or spread over several.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "galn_host_internal.h"

namespace {

double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Chunk {                         // results of reads [r0, r0 + m) of a request
    int r0 = 0, m = 0;
    galn::hvec<int32_t> n_aln;
    galn::hvec<galn_aln1> rec;
    galn::hvec<uint64_t> pops, trace;
};

struct Request {
    int64_t id = 0;
    uint64_t need = 0;                 // device memory its search stacks need (request_stack_need)
    int64_t admit_seq = -1;            // order of admission
    galn_opts opt;
    std::vector<char> seq;
    std::vector<int64_t> off;
    std::vector<int32_t> batch;        // own bwa batch of each read
    std::vector<int32_t> bmax;         // longest read of each own batch
    int n = 0, next = 0, done_reads = 0;
    std::vector<Chunk> chunks;         // finished pieces, in any order
    // results, in read order (assembled when the last piece is done)
    galn::hvec<int32_t> n_aln;
    galn::hvec<galn_aln1> rec;
    galn::hvec<uint64_t> pops, trace;
    double t_submit = 0, t_done = 0;
    int rc = 0;
    bool done = false;
    galn_results res;
};

}  // namespace

struct galn_server {
    galn_index *ix = nullptr;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;       // submitted, not yet admitted
    std::vector<Request *> active;     // admitted, not finished
    std::map<int64_t, Request *> all;
    int64_t next_id = 1;
    bool stop = false;
    size_t max_queued = 1 << 16;
    int max_active = 64;
    int step_reads = 1 << 18;
    int fill_reads = 0;                // with a step running, wait for this many reads before the next (0: start at once)
    int running = 0;                   // steps on the device now
    int n_workers = 2;
    std::vector<galn::ExecCtx *> ctxs;
    std::vector<std::thread> workers;
    // admission by stack memory
    uint64_t mem_budget = 0;           // device memory the admitted requests' stacks may take
    uint64_t mem_active = 0, mem_peak = 0;
    int head_passed = 0;               // requests admitted past the queue's head while it did not fit
    int64_t held_back = 0;             // times a queued request was passed over for lack of stack memory
    int64_t admitted = 0;
    std::vector<int64_t> admit_order;  // request ids in the order they were admitted (finished requests)
    // statistics
    std::vector<double> lat_ms;
    int64_t reads_done = 0, steps = 0;
    double busy_ms = 0;
};

namespace {

constexpr int kMaxBypass = 64;         // later requests admitted past one that does not fit, at most

// The device memory the search stacks of a request need: a first-tier stack for each of its reads in
// flight (reads of a step), as the first tier sizes one (entries and links, a head per score bucket, the
// width arrays of the longest read, the records), and the deepest stack one of its reads may build, an arena
// that holds the max_entries cut-off (the heavy-read tier's; the reference sizes its arenas the same way,
// src/galn.cu:916-918). n_stacks, max_diff and the entry width follow the options as the engine derives them
// (src/aln_host.c:23-38).
uint64_t request_stack_need(const galn_index *ix, const galn_opts *o, int n, int max_len, int step_reads)
{
    int max_diff = o->max_diff, max_gapo = o->max_gapo;
    if (o->fnr > 0.0) max_diff = galn_cal_maxdiff(max_len, 0.02, o->fnr);
    if (max_diff < max_gapo) max_gapo = max_diff;
    const int64_t n_stacks = std::max<int64_t>(1, (int64_t)(max_diff + 1) * o->s_mm + (int64_t)(max_gapo + 1) * o->s_gapo +
                                                      (int64_t)(o->max_gape + 1) * o->s_gape);
    const bool wide = max_diff > 125 || max_gapo > 126 || o->max_gape > 126 || ix->dev.seq_len >= (1ull << 38);
    const uint64_t esz = (wide ? 32 : 16) + 4;
    const int seed = o->seed_len >= 0 && o->seed_len < max_len ? o->seed_len + 1 : 0;
    const uint64_t slot = (uint64_t)ix->t0_cap * esz + (uint64_t)n_stacks * 4 + (uint64_t)(max_len + 2 + seed) * 8 +
                          (uint64_t)ix->t0_aln * 24;
    const uint64_t deepest = ((uint64_t)std::max(o->max_entries, 0) + 16) * esz + (uint64_t)n_stacks * 4;
    return (uint64_t)std::min(n, step_reads) * slot + (n > 0 ? deepest : 0);
}

}  // namespace

// Moves queued requests into the active set while their stack memory fits (and max_active allows); a
// request that does not fit is passed by later ones up to kMaxBypass times. Returns whether any was admitted.
static bool admit(galn_server *s, bool dry_run)
{
    bool any = false;
    int passed = s->head_passed;
    uint64_t used = s->mem_active;
    size_t n_active = s->active.size();
    for (size_t q = 0; q < s->queue.size() && (int)n_active < s->max_active;) {
        Request *rq = s->queue[q];
        const bool fits = n_active == 0 || used + rq->need <= s->mem_budget;
        if (!fits) {
            if (q == 0 && passed >= kMaxBypass) break;   // the head has waited long enough: nothing passes it
            if (!dry_run) ++s->held_back;
            ++q;
            continue;
        }
        any = true;
        used += rq->need;
        ++n_active;
        if (q > 0) ++passed;
        if (dry_run) { ++q; continue; }
        if (q == 0) passed = 0;
        rq->admit_seq = s->admitted++;
        if (s->admit_order.size() < ((size_t)1 << 20)) s->admit_order.push_back(rq->id);
        s->active.push_back(rq);
        s->queue.erase(s->queue.begin() + (long)q);
    }
    if (!dry_run) {
        s->head_passed = passed;
        s->mem_active = used;
        s->mem_peak = std::max(s->mem_peak, used);
    }
    return any;
}

static void finish_request(Request *rq)
{
    std::sort(rq->chunks.begin(), rq->chunks.end(), [](const Chunk &a, const Chunk &b) { return a.r0 < b.r0; });
    for (auto &c : rq->chunks) {
        rq->n_aln.insert(rq->n_aln.end(), c.n_aln.begin(), c.n_aln.end());
        rq->rec.insert(rq->rec.end(), c.rec.begin(), c.rec.end());
        rq->pops.insert(rq->pops.end(), c.pops.begin(), c.pops.end());
        rq->trace.insert(rq->trace.end(), c.trace.begin(), c.trace.end());
    }
    std::vector<Chunk>().swap(rq->chunks);
    auto *P = new galn::ResultsPriv();
    P->n_aln.swap(rq->n_aln);
    P->rec.swap(rq->rec);
    P->pops.swap(rq->pops);
    P->trace.swap(rq->trace);
    P->rec_off.resize((size_t)rq->n + 1);
    int64_t t = 0;
    for (int r = 0; r < rq->n; ++r) {
        P->rec_off[r] = t;
        if (P->n_aln[r] > 0) t += P->n_aln[r];
    }
    P->rec_off[rq->n] = t;
    if (P->rec.empty()) P->rec.resize(1);
    if (P->n_aln.empty()) { P->n_aln.resize(1); P->pops.resize(1); P->trace.resize(1); }
    rq->res.n_reads = rq->n;
    rq->res.n_aln = P->n_aln.data();
    rq->res.rec_offset = P->rec_off.data();
    rq->res.rec = P->rec.data();
    rq->res.n_pops = P->pops.data();
    rq->res.trace = P->trace.data();
    rq->res._priv = P;
    std::vector<char>().swap(rq->seq);
}

static void serve_loop(galn_server *s, galn::ExecCtx *ctx)
{
    struct Piece { Request *rq; int r0, m; };
    std::vector<char> seq;
    std::vector<int64_t> off;
    std::vector<int32_t> batch, bmax, bset;
    std::vector<galn_opts> sets;
    for (;;) {
        std::vector<Piece> pieces;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            // wait for reads nobody has taken yet (a request may be active with all its reads in flight)
            auto has_work = [&] {
                for (Request *rq : s->active)
                    if (rq->next < rq->n || (rq->n == 0 && rq->next == 0)) return true;
                return !s->queue.empty() && admit(s, true);
            };
            // with a step already running, a fill target makes the next step wait until it can take that
            // many reads (or the running step ends): fewer, fuller steps when requests arrive quickly
            auto can_start = [&] {
                if (s->running == 0 || s->fill_reads == 0) return true;
                int64_t avail = 0;
                for (Request *rq : s->active) avail += std::max(0, rq->n - rq->next);
                for (size_t q = 0; q < s->queue.size() && (int)s->active.size() + (int)q < s->max_active; ++q)
                    avail += s->queue[q]->n;
                return avail >= std::min(s->fill_reads, s->step_reads);
            };
            s->cv_work.wait(lk, [&] { return s->stop || (has_work() && can_start()); });
            if (s->stop && !has_work()) return;
            admit(s, false);
            // equal shares first, then the oldest requests take what is left
            int budget = s->step_reads;
            int na = (int)s->active.size();
            int share = std::max(4096, s->step_reads / std::max(1, na));
            std::vector<int> take(na, 0);
            for (int a = 0; a < na && budget > 0; ++a) {
                Request *rq = s->active[a];
                int m = std::min({std::max(0, rq->n - rq->next), share, budget});
                take[a] = m;
                budget -= m;
            }
            for (int a = 0; a < na && budget > 0; ++a) {
                Request *rq = s->active[a];
                int m = std::min(std::max(0, rq->n - rq->next - take[a]), budget);
                take[a] += m;
                budget -= m;
            }
            for (int a = 0; a < na; ++a) {
                Request *rq = s->active[a];
                if (take[a] > 0 || (rq->n == 0 && rq->next == 0)) {
                    pieces.push_back({rq, rq->next, take[a]});
                    rq->next += take[a];
                    if (rq->n == 0) rq->next = 1;   // an empty request is taken once
                }
            }
            if (!pieces.empty()) ++s->running;
        }
        if (pieces.empty()) continue;
        // one combined job: every request is one option set, every (request, own batch) one batch
        seq.clear(); off.clear(); batch.clear(); bmax.clear(); bset.clear(); sets.clear();
        off.push_back(0);
        for (size_t p = 0; p < pieces.size(); ++p) {
            Request *rq = pieces[p].rq;
            const int r0 = pieces[p].r0, r1 = pieces[p].r0 + pieces[p].m;
            sets.push_back(rq->opt);
            std::map<int, int> gb;   // own batch -> batch of the step
            const int64_t sbase = (int64_t)seq.size() - (r1 > r0 ? rq->off[r0] : 0);
            if (r1 > r0) seq.insert(seq.end(), rq->seq.begin() + rq->off[r0], rq->seq.begin() + rq->off[r1]);
            int last_own = -1, last_step = -1;
            for (int r = r0; r < r1; ++r) {
                const int own = rq->batch[r];
                if (own != last_own) {
                    auto it = gb.find(own);
                    if (it == gb.end()) {
                        it = gb.emplace(own, (int)bmax.size()).first;
                        bmax.push_back(rq->bmax[own]);
                        bset.push_back((int32_t)p);
                    }
                    last_own = own;
                    last_step = it->second;
                }
                off.push_back(sbase + rq->off[r + 1]);
                batch.push_back(last_step);
            }
        }
        galn_reads in;
        memset(&in, 0, sizeof(in));
        in.n_reads = (int32_t)batch.size();
        in.seq = seq.empty() ? "" : seq.data();
        in.offset = off.data();
        in.batch = batch.data();
        in.batch_max_len = bmax.data();
        in.n_batches = (int32_t)bmax.size();
        galn_results res;
        memset(&res, 0, sizeof(res));
        int rc = 0;
        double t0 = now_ms();
        if (in.n_reads > 0) {
            rc = galn::run_job_multi(s->ix, *ctx, sets.data(), (int)sets.size(), bset.data(), &in, GALN_ENGINE_PERSISTENT,
                                     &res);
        }
        double t1 = now_ms();
        // each piece's results, copied outside the lock (the step's results are in read order)
        std::vector<Chunk> chunks(pieces.size());
        {
            int j = 0;
            for (size_t p = 0; p < pieces.size(); ++p) {
                Chunk &ch = chunks[p];
                const int m = pieces[p].m;
                ch.r0 = pieces[p].r0; ch.m = m;
                if (rc) {
                    ch.n_aln.assign((size_t)m, GALN_ERR_STACK);
                    ch.pops.assign((size_t)m, 0);
                    ch.trace.assign((size_t)m, 0);
                } else if (m > 0) {
                    ch.n_aln.assign(res.n_aln + j, res.n_aln + j + m);
                    ch.pops.assign(res.n_pops + j, res.n_pops + j + m);
                    ch.trace.assign(res.trace + j, res.trace + j + m);
                    ch.rec.assign(res.rec + res.rec_offset[j], res.rec + res.rec_offset[j + m]);
                }
                j += m;
            }
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->busy_ms += t1 - t0;
            ++s->steps;
            --s->running;
            for (size_t p = 0; p < pieces.size(); ++p) {
                auto &pc = pieces[p];
                Request *rq = pc.rq;
                rq->chunks.push_back(std::move(chunks[p]));
                if (rc) rq->rc = rc;
                rq->done_reads += pc.m;
                s->reads_done += pc.m;
                if (rq->done_reads >= rq->n) {
                    finish_request(rq);
                    rq->t_done = now_ms();
                    rq->done = true;
                    s->lat_ms.push_back(rq->t_done - rq->t_submit);
                    s->active.erase(std::find(s->active.begin(), s->active.end(), rq));
                    s->mem_active -= rq->need;
                }
            }
        }
        if (in.n_reads > 0 && rc == 0) galn_results_free(&res);
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

extern "C" galn_server *galn_server_start(galn_index *ix, size_t stack_bytes, int *err)
{
    if (!ix) { if (err) *err = GALN_EINVAL; return nullptr; }
    auto *s = new galn_server();
    s->ix = ix;
    if (cudaSetDevice(ix->dev.device) != cudaSuccess) { delete s; if (err) *err = GALN_ECUDA; return nullptr; }
    s->mem_budget = stack_bytes;
    if (!stack_bytes) {   // default: half of the device memory free now (the index is already resident)
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { delete s; if (err) *err = GALN_ECUDA; return nullptr; }
        s->mem_budget = free_b / 2;
    }
    for (int w = 0; w < s->n_workers; ++w) {
        auto *c = new galn::ExecCtx();
        c->mem_share = 1.0 / s->n_workers;
        if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
            if (err) *err = GALN_ECUDA;
            for (auto *q : s->ctxs) { cudaStreamDestroy(q->stream); delete q; }
            delete c;
            delete s;
            return nullptr;
        }
        galn::index_l2_policy(ix, c->stream, ix->occ);
        c->l2_occ = ix->occ;
        s->ctxs.push_back(c);
    }
    for (auto *c : s->ctxs) s->workers.emplace_back(serve_loop, s, c);
    if (err) *err = 0;
    return s;
}

extern "C" int galn_server_configure(galn_server *s, int step_reads, int max_active)
{
    if (!s || step_reads < 1024 || max_active < 1) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    s->step_reads = step_reads;
    s->max_active = max_active;
    return 0;
}

extern "C" int galn_server_set_step_fill(galn_server *s, int fill_reads)
{
    if (!s || fill_reads < 0) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    s->fill_reads = fill_reads;
    s->cv_work.notify_all();
    return 0;
}

extern "C" int galn_server_stop(galn_server *s)
{
    if (!s) return GALN_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    cudaSetDevice(s->ix->dev.device);
    for (auto *c : s->ctxs) {
        c->release();
        cudaStreamDestroy(c->stream);
        delete c;
    }
    for (auto &kv : s->all) {
        if (kv.second->done) galn_results_free(&kv.second->res);
        delete kv.second;
    }
    delete s;
    return 0;
}

extern "C" int64_t galn_aln_submit(galn_server *s, const galn_opts *o, const galn_reads *in)
{
    if (!s || !o || !in || in->n_reads < 0 || (in->n_reads > 0 && (!in->seq || !in->offset))) return GALN_EINVAL;
    auto *rq = new Request();
    rq->opt = *o;
    const int n = in->n_reads;
    rq->n = n;
    int64_t base = n ? in->offset[0] : 0, total = n ? in->offset[n] - base : 0;
    rq->seq.assign(in->seq + base, in->seq + base + total);
    rq->off.resize((size_t)n + 1);
    int nb = 0;
    rq->batch.resize((size_t)n);
    for (int r = 0; r <= n; ++r) rq->off[r] = in->offset[r] - base;
    for (int r = 0; r < n; ++r) {
        int64_t len = rq->off[r + 1] - rq->off[r];
        int b = in->batch ? in->batch[r] : r / galn::kBatchReads;
        if (len < 0 || len > 65535 || b < 0) { delete rq; return GALN_EINVAL; }
        rq->batch[r] = b;
        nb = std::max(nb, b + 1);
    }
    if (in->batch_max_len) nb = std::max(nb, (int)in->n_batches);
    rq->bmax.assign((size_t)std::max(nb, 1), 0);
    for (int r = 0; r < n; ++r) rq->bmax[rq->batch[r]] = std::max(rq->bmax[rq->batch[r]], (int32_t)(rq->off[r + 1] - rq->off[r]));
    if (in->batch_max_len)
        for (int b = 0; b < in->n_batches; ++b) rq->bmax[b] = std::max(rq->bmax[b], in->batch_max_len[b]);
    rq->n_aln.reserve((size_t)n);
    rq->pops.reserve((size_t)n);
    rq->trace.reserve((size_t)n);
    const int max_len = n ? *std::max_element(rq->bmax.begin(), rq->bmax.end()) : 0;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->queue.size() >= s->max_queued) { delete rq; return GALN_EBUSY; }
    rq->need = request_stack_need(s->ix, o, n, max_len, s->step_reads);
    rq->id = s->next_id++;
    rq->t_submit = now_ms();
    s->all[rq->id] = rq;
    s->queue.push_back(rq);
    s->cv_work.notify_one();
    return rq->id;
}

extern "C" int galn_aln_wait(galn_server *s, int64_t id, int timeout_ms, galn_results *out)
{
    if (!s || !out) return GALN_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return GALN_EINVAL;
    Request *rq = it->second;
    auto ready = [&] { return rq->done; };
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return GALN_ETIMEOUT;
    int rc = rq->rc;
    *out = rq->res;              // the caller owns the results now (galn_results_free)
    s->all.erase(it);
    delete rq;
    return rc;
}

extern "C" int galn_stack_need(galn_server *s, const galn_opts *o, const galn_reads *in, uint64_t *bytes)
{
    if (!s || !o || !in || !bytes || in->n_reads < 0 || (in->n_reads > 0 && !in->offset)) return GALN_EINVAL;
    int max_len = 0;
    for (int r = 0; r < in->n_reads; ++r) max_len = std::max<int64_t>(max_len, in->offset[r + 1] - in->offset[r]);
    if (in->batch_max_len)
        for (int b = 0; b < in->n_batches; ++b) max_len = std::max(max_len, (int)in->batch_max_len[b]);
    std::lock_guard<std::mutex> lk(s->mu);
    *bytes = request_stack_need(s->ix, o, in->n_reads, max_len, s->step_reads);
    return 0;
}

extern "C" int galn_server_memory(galn_server *s, uint64_t *budget, uint64_t *in_use, uint64_t *peak, int64_t *held_back)
{
    if (!s) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if (budget) *budget = s->mem_budget;
    if (in_use) *in_use = s->mem_active;
    if (peak) *peak = s->mem_peak;
    if (held_back) *held_back = s->held_back;
    return 0;
}

extern "C" int galn_server_admissions(galn_server *s, int64_t *ids, int n)
{
    if (!s || n < 0 || (n > 0 && !ids)) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    const int k = (int)std::min<size_t>((size_t)n, s->admit_order.size());
    for (int i = 0; i < k; ++i) ids[i] = s->admit_order[(size_t)i];
    return k;
}

extern "C" int galn_server_stats(galn_server *s, double *p50_ms, double *p99_ms, int64_t *n_requests, int64_t *n_reads,
                                 double *busy_ms, int64_t *steps)
{
    if (!s) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) { return v.empty() ? 0.0 : v[(size_t)std::min<double>(v.size() - 1, floor(q * (v.size() - 1) + 0.5))]; };
    if (p50_ms) *p50_ms = pct(0.50);
    if (p99_ms) *p99_ms = pct(0.99);
    if (n_requests) *n_requests = (int64_t)v.size();
    if (n_reads) *n_reads = s->reads_done;
    if (busy_ms) *busy_ms = s->busy_ms;
    if (steps) *steps = s->steps;
    return 0;
}
