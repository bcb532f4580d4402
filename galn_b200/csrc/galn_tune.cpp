// galn_tune.cpp -- the autotuner: per option set, the occurrence layout, the first tier's stack depth and
// block size.
//
// The first tier's stack depth decides the split between the thread-per-read and the warp-per-read tiers:
// a read whose search needs more stack than that leaves the thread tier and is searched by a warp. The
// best depth depends on the options (how many reads backtrack deeply) and on the index (how long
// exact-match chains run), so it is measured: a sample of the job's reads is searched once per candidate
// (layout x depth x block size) and the fastest device time wins. The layout (64 or 80 symbols per 32-byte
// block) trades index size, which decides how much of it stays in L2, against popcounts per lookup. A second
// stage, with that choice fixed, times the warp tier's stack arena per warp and its count of big-arena warps
// (the warps that take reads outgrowing a small arena). Results never depend on the choice; only speed does.
// The table is keyed by the option block, so every parameter set has its own entry.
#include <string.h>

#include <algorithm>
#include <vector>

#include "galn_host_internal.h"

namespace galn {

uint64_t opts_key(const galn_opts *o)
{
    // FNV-1a over the option block (n_threads is only a header value and does not change the search)
    galn_opts c = *o;
    c.n_threads = 0;
    const unsigned char *p = (const unsigned char *)&c;
    uint64_t h = 1469598103934665603ULL;
    for (size_t i = 0; i < sizeof(c); ++i) h = (h ^ p[i]) * 1099511628211ULL;
    return h;
}

}  // namespace galn

using namespace galn;

extern "C" int galn_autotune(galn_index *ix, const galn_opts *o, const galn_reads *in, int max_sample, int *best_cap,
                             int *best_block, int *best_occ, double *best_ms)
{
    if (!ix || !o || !in || in->n_reads < 0) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    galn_reads s = *in;
    if (max_sample > 0 && s.n_reads > max_sample) s.n_reads = max_sample;
    static const int caps[] = {256, 512, 1024, 2048, 4096};
    static const int blocks[] = {128, 256};
    static const int layouts[] = {64, 80};
    // the warp tier's arena per warp (64-entry chunks) and its count of big-arena warps, timed with the
    // first stage's choice. Only sizes at or above the defaults: a sample holds fewer of the heaviest reads
    // than the whole input, and smaller arenas or fewer big warps that suit the sample choke on the whole
    // (2048 chunks and 64 big warps ran the aDNA sample fastest and the full 2 M reads 2.3x slower).
    static const int arenas[] = {8192, 16384};
    static const int bigs[] = {128, 256};
    const int saved_cap = ix->t0_cap, saved_block = ix->t0_block, saved_occ = ix->occ;
    const int saved_arena = ix->warp_arena, saved_big = ix->warp_big, saved_div = ix->fused_div;
    const bool saved_stats = ix->keep_stats, saved_fused = ix->use_fused;
    ix->keep_stats = false;
    int bc = saved_cap, bb = saved_block, bo = saved_occ, ba = saved_arena, bg = saved_big;
    int bd = saved_fused ? saved_div : 0;
    double bms = 1e300;
    int rc = 0;
    auto time_one = [&](double &ms) {
        ix->tune_active = true;
        galn_results res;
        memset(&res, 0, sizeof(res));
        int r = run_job(ix, ix->main, o, &s, GALN_ENGINE_PERSISTENT, &res);
        ix->tune_active = false;
        if (r) return r;
        galn_results_free(&res);
        ms = ix->main.last.ms_device;
        return 0;
    };
    for (int occ : layouts)
        for (int cap : caps)
            for (int blk : blocks) {
                if (rc) break;
                ix->t0_cap = cap;
                ix->t0_block = blk;
                ix->occ = occ;
                double ms = 0;
                rc = time_one(ms);
                if (!rc && ms < bms) { bms = ms; bc = cap; bb = blk; bo = occ; }
            }
    ix->t0_cap = bc;
    ix->t0_block = bb;
    ix->occ = bo;
    for (int ar : arenas)
        for (int bg2 : bigs) {
            if (rc) break;
            ix->warp_arena = ar;
            ix->warp_big = bg2;
            double ms = 0;
            rc = time_one(ms);
            if (!rc && ms < bms) { bms = ms; ba = ar; bg = bg2; }
        }
    // the launch form: two launches (0) or the fused launch with 1/16 .. 1/2 of its blocks warp-tier warps
    // from the start
    {
        static const int divs[] = {0, 16, 8, 4, 2};
        ix->warp_arena = ba;
        ix->warp_big = bg;
        ix->use_fused = true;
        for (int dv : divs) {
            if (rc) break;
            ix->fused_div = dv;
            double ms = 0;
            rc = time_one(ms);
            if (!rc && ms < bms) { bms = ms; bd = dv; }
        }
    }
    ix->t0_cap = saved_cap;
    ix->t0_block = saved_block;
    ix->occ = saved_occ;
    ix->warp_arena = saved_arena;
    ix->warp_big = saved_big;
    ix->fused_div = saved_div;
    ix->use_fused = saved_fused;
    ix->keep_stats = saved_stats;
    if (rc) return rc;
    ix->tuned[opts_key(o)] = galn_index::TuneChoice{bc, bb, bo, ba, bg, bd};
    if (best_cap) *best_cap = bc;
    if (best_block) *best_block = bb;
    if (best_occ) *best_occ = bo;
    if (best_ms) *best_ms = bms;
    return 0;
}

extern "C" int galn_autotune_choice(galn_index *ix, const galn_opts *o, int *cap, int *block, int *occ,
                                    int *warp_arena, int *warp_big, int *fused_div)
{
    if (!ix || !o) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    auto it = ix->tuned.find(opts_key(o));
    if (it == ix->tuned.end()) return GALN_EINVAL;
    if (cap) *cap = it->second.cap;
    if (block) *block = it->second.block;
    if (occ) *occ = it->second.occ;
    if (warp_arena) *warp_arena = it->second.arena;
    if (warp_big) *warp_big = it->second.big;
    if (fused_div) *fused_div = it->second.fused_div;
    return 0;
}

extern "C" int galn_autotune_clear(galn_index *ix)
{
    if (!ix) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    ix->tuned.clear();
    return 0;
}
