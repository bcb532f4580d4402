// galn_serve.cpp -- the request loop around a resident index.
//
// galn_aln_submit copies a request (its own options and bwa batch boundaries) into a queue; a worker thread
// takes requests in arrival order and runs them on the index. galn_aln_wait blocks until a request's
// results are ready. Each request's results are computed exactly as by galn_aln_run_batch of that request
// alone (the per-batch options come only from the request's own reads), so they do not depend on what else
// is queued.
#include <string.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "galn_host_internal.h"

namespace {

struct Request {
    int64_t id = 0;
    galn_opts opt;
    std::vector<char> seq;
    std::vector<int64_t> off;
    std::vector<int32_t> batch;
    std::vector<int32_t> bmax;
    int rc = 0;
    bool done = false;
    galn_results res;
};

}  // namespace

struct galn_server {
    galn_index *ix = nullptr;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::map<int64_t, Request *> all;
    int64_t next_id = 1;
    bool stop = false;
    size_t max_queued = 4096;
    std::thread worker;
};

static void serve_loop(galn_server *s)
{
    for (;;) {
        Request *rq = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
            if (s->queue.empty()) return;
            rq = s->queue.front();
            s->queue.pop_front();
        }
        galn_reads in;
        memset(&in, 0, sizeof(in));
        in.n_reads = (int32_t)rq->off.size() - 1;
        in.seq = rq->seq.data();
        in.offset = rq->off.data();
        in.batch = rq->batch.empty() ? nullptr : rq->batch.data();
        in.batch_max_len = rq->bmax.empty() ? nullptr : rq->bmax.data();
        in.n_batches = (int32_t)rq->bmax.size();
        memset(&rq->res, 0, sizeof(rq->res));
        int rc = galn_aln_run_batch(s->ix, &rq->opt, &in, GALN_ENGINE_PERSISTENT, &rq->res);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            rq->rc = rc;
            rq->done = true;
            std::vector<char>().swap(rq->seq);
        }
        s->cv_done.notify_all();
    }
}

extern "C" galn_server *galn_server_start(galn_index *ix, size_t stack_bytes, int *err)
{
    (void)stack_bytes;
    if (!ix) { if (err) *err = GALN_EINVAL; return nullptr; }
    auto *s = new galn_server();
    s->ix = ix;
    s->worker = std::thread(serve_loop, s);
    if (err) *err = 0;
    return s;
}

extern "C" int galn_server_stop(galn_server *s)
{
    if (!s) return GALN_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->worker.join();
    for (auto &kv : s->all) {
        if (kv.second->done && kv.second->rc == 0) galn_results_free(&kv.second->res);
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
    int n = in->n_reads;
    int64_t base = n ? in->offset[0] : 0, total = n ? in->offset[n] - base : 0;
    rq->seq.assign(in->seq + base, in->seq + base + total);
    rq->off.resize((size_t)n + 1);
    for (int r = 0; r <= n; ++r) rq->off[r] = in->offset[r] - base;
    if (in->batch) rq->batch.assign(in->batch, in->batch + n);
    if (in->batch_max_len) rq->bmax.assign(in->batch_max_len, in->batch_max_len + in->n_batches);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->queue.size() >= s->max_queued) { delete rq; return GALN_EBUSY; }
    rq->id = s->next_id++;
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
    if (rc == 0) *out = rq->res;
    s->all.erase(it);
    delete rq;
    return rc;
}
