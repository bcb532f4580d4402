// galn_warp.cuh -- the heavy-read tier: one warp per read, up to 32 stack entries expanded at once.
//
// Why this is exact. With positive penalties (s_mm, s_gapo, s_gape > 0) every child of an entry popped from
// score bucket b goes to a bucket above b, except the exact-match child, which has score b and is pushed
// last, so it is the very next pop (src/bwtgap_hd.h:457-470 push order). Bucket b therefore receives no
// entry while it is being popped: its pops are the entries e_m, e_{m-1}, ..., e_1 (LIFO), each followed
// by its chain of exact-match children. Between two hits the expansion of a chain depends only on its
// first entry, the width arrays and max_diff, none of which change without a hit; so the chains of the
// top W <= 32 entries of bucket b can be expanded at the same time, one per lane.
//
// One wave: lane j takes the j-th entry from the top of bucket b (lane 0 takes a pending exact child left
// by the previous wave), runs its chain for up to kWR pops, staging the pushes of each pop (in the order
// bwt_match_gap pushes them) in global memory, one list per distinct target bucket (b+s_mm, b+s_gapo,
// b+s_gape), with 4 bytes of per-pop data in shared memory, and stopping at a hit (a "hazard"). Then the warp replays the
// lanes in order exactly as the sequential search would pop them: the max_entries test before each pop,
// n_entries after each pop and push, the pop count, the trace hash, the first hit (handled sequentially:
// best_score, max_diff, -R, gapped-hit de-duplication, gap_shadow, the record). Replay stops at a hit or at a
// lane whose chain is not finished; later lanes' speculation is discarded and their entries stay on the stack.
// The pushes of the replayed pops are committed to their buckets in replay order (per bucket: lane order,
// then pop order), so every bucket is the same LIFO as in the sequential search.
//
// Storage: each bucket is a chain of 32-entry chunks in the warp's arena (global memory), with its top
// chunk, fill and entry count in shared memory. Widths, the query and the per-pop data are in shared
// memory; staged pushes (and, in trace mode, popped entries) in a per-warp global staging area. Reads the tier cannot take (length > 256, n_stacks > 256, a penalty <= 0, 32-byte entries) or
// that outgrow the arena or the record buffer go to the thread tiers (the host routes them).
#pragma once

#include "galn_search.cuh"

namespace galn {

constexpr int kWMaxB = 256;      // buckets
constexpr int kWMaxLen = 256;    // read length
constexpr int kWR = 32;          // pops per lane per wave
constexpr int kWL = 128;         // staged pushes per lane and target list per wave
constexpr int kWCH = 32;         // entries per chunk
constexpr int kWNewC = (kWCH + 32 * kWL) / kWCH + 2;   // chunks one commit may allocate

struct WarpSmem {
    int32_t top_chunk[kWMaxB];
    int32_t n_in[kWMaxB];
    uint16_t top_cnt[kWMaxB];
    uint32_t mask[kWMaxB / 32];
    uint64_t W[kWMaxLen + 1];
    uint64_t SW[kWMaxLen + 1];
    uint8_t q[kWMaxLen];
    // per pop of each lane: pushes (bits 0-7, the fused exact child not counted), has an exact child
    // (bit 8), index blocks read (bits 16-31)
    uint32_t meta[32][kWR + 1];       // one word of padding per row: lanes writing the same pop hit distinct banks
    uint4 hz[32];                     // hazard entry of each lane
    uint64_t hk[32], hl[32];          // its interval after the exact tail
    int32_t lane_np[32], lane_end[32];
    uint32_t lane_nl[32][3];          // staged pushes of each lane per target list
    uint4 lane_x[32];                 // pending exact child of a lane that stopped mid-chain
    int32_t newc[kWNewC];             // chunks allocated for one commit
    int32_t incl[32];                 // inclusive scan of the lanes' counts in one commit
};

struct WArgs {
    IndexView ix;
    const uint8_t *query;
    const int64_t *off;
    const int32_t *bidx;
    const int32_t *maxdiff;
    const BatchOpt *bopt;
    int seed_len;
    const int32_t *list;
    int n;
    int32_t *claim;
    int n_warps;
    uint4 *chunks;            // n_warps * arena_chunks * kWCH entries
    int32_t *chunk_prev;      // n_warps * arena_chunks
    int32_t *free_ids;        // n_warps * arena_chunks
    int arena_chunks;
    uint64_t *aln;            // n_warps * aln_cap * 3
    int aln_cap;
    uint4 *stage;             // n_warps * 3 lists * 32 lanes * kWL staged pushes
    uint4 *prec;              // n_warps * 32 lanes * kWR popped entries (trace mode)
    int32_t *out_n;
    int64_t *out_off;
    uint64_t *out_pops, *out_trace;
    int32_t *out_peak;
    uint32_t *out_fetch;
    int8_t *out_tier;
    int tier;
    uint64_t *out_rec;
    unsigned long long *rec_top;
    int64_t rec_cap;
    int32_t *ovf;
    int32_t *ovf_n;
    unsigned long long *dbg;  // optional counters (kWDbg entries), or NULL
};

// optional counters of the warp tier (per launch, summed over warps)
enum { kDbgReads, kDbgWaves, kDbgLanes, kDbgConsumed, kDbgPops, kDbgCont, kDbgHazard, kDbgCycChain,
       kDbgCycReplay, kDbgCycCommit, kDbgCycLoad, kDbgChainPops, kWDbg };

// an entry in registers (the score is the bucket of the wave)
struct WEnt {
    uint64_t k, l;
    int i, isdiff, n_mm, n_gapo, n_gape, n_ins, state;
};

__device__ __forceinline__ uint4 wpack(const WEnt &x)
{
    uint64_t w0 = (x.k & kK38) | ((uint64_t)(uint32_t)x.i << 38) | ((uint64_t)(x.n_mm & 127) << 54)
                | ((uint64_t)x.state << 61) | ((uint64_t)(x.isdiff ? 1 : 0) << 63);
    uint64_t w1 = (x.l & kK38) | ((uint64_t)(x.n_gapo & 127) << 38) | ((uint64_t)(x.n_gape & 127) << 45)
                | ((uint64_t)(x.n_ins & 255) << 52);
    return make_uint4((uint32_t)w0, (uint32_t)(w0 >> 32), (uint32_t)w1, (uint32_t)(w1 >> 32));
}

__device__ __forceinline__ WEnt wunpack(uint4 v)
{
    uint64_t w0 = (uint64_t)v.x | ((uint64_t)v.y << 32), w1 = (uint64_t)v.z | ((uint64_t)v.w << 32);
    WEnt x;
    x.k = w0 & kK38;
    x.i = (int)((w0 >> 38) & 0xffff);
    x.n_mm = (int)((w0 >> 54) & 127);
    x.state = (int)((w0 >> 61) & 3);
    x.isdiff = (int)(w0 >> 63);
    x.l = w1 & kK38;
    x.n_gapo = (int)((w1 >> 38) & 127);
    x.n_gape = (int)((w1 >> 45) & 127);
    x.n_ins = (int)((w1 >> 52) & 255);
    return x;
}

__device__ __forceinline__ uint4 wpack_child(uint64_t k, uint64_t l, int i, int n_mm, int n_gapo, int n_gape, int n_ins,
                                             int state, int isdiff)
{
    WEnt x;
    x.k = k; x.l = l; x.i = i; x.isdiff = isdiff; x.n_mm = n_mm; x.n_gapo = n_gapo; x.n_gape = n_gape;
    x.n_ins = n_ins; x.state = state;
    return wpack(x);
}

struct WCtx {
    int len, max_diff, max_diff0, use_seed, seed_len_r;
    bool gape, nonstop;
};

// one lane's chain: end code 0 = finished, 1 = hazard (a hit) at its last pop, 2 = stopped with x pending,
// 3 = its last pop pushes a score >= n_stacks (bwt_match_gap returns BWTGAP_ERR_SCORE there).
// st: this lane's three staging lists (kWL apart, 32 * kWL between lists); tl: list of each push kind
// (mismatch, gap open, gap extension); pr: this lane's popped-entry records (trace mode)
template <bool TRACE>
__device__ __forceinline__ void lane_chain(const IndexView &ix, const BatchOpt &O, const WCtx &c, WarpSmem *S, int lane,
                                           WEnt x, int b, uint32_t &fetches, uint4 *st, const int tl[3], uint4 *pr)
{
    int np = 0, endc = 0;
    int nl0 = 0, nl1 = 0, nl2 = 0;
    const size_t lstride = (size_t)32 * kWL;
    // a push of the given kind (0 mismatch, 1 gap open, 2 gap extension); a score at or past n_stacks ends
    // the read
#define WPUSH(KIND, BKT, ...)                                                           \
    do {                                                                                \
        int bk_ = (BKT);                                                                \
        if (bk_ >= O.n_stacks) { err = true; break; }                                   \
        int L_ = tl[KIND];                                                              \
        int &n_ = L_ == 0 ? nl0 : (L_ == 1 ? nl1 : nl2);                                \
        st[L_ * lstride + n_] = wpack_child(__VA_ARGS__);                               \
        ++n_;                                                                           \
        ++npu;                                                                          \
    } while (0)
    for (;;) {
        bool err = false;
        const uint32_t f_pop = fetches;
        if (TRACE) pr[np] = wpack(x);
        int diffs = x.n_mm + x.n_gapo + (c.gape ? x.n_gape : 0);
        int m = c.max_diff - diffs;
        int i = x.i;
        uint32_t npu = 0, hx = 0;
        if (m < 0 || (i > 0 && m < (int)(S->W[i - 1] >> 48))) {
            S->meta[lane][np] = 0; ++np; endc = 0; break;
        }
        if (i == 0) {
            S->hz[lane] = wpack(x); S->hk[lane] = x.k; S->hl[lane] = x.l;
            S->meta[lane][np] = 0; ++np; endc = 1; break;
        }
        if (m == 0 && (x.state == kStM || c.gape || x.n_gape == O.max_gape)) {
            uint64_t k = x.k, l = x.l;
            if (match_exact_alt(ix, i, S->q, k, l, fetches)) {
                S->hz[lane] = wpack(x); S->hk[lane] = k; S->hl[lane] = l; endc = 1;
            } else endc = 0;
            S->meta[lane][np] = (fetches - f_pop) << 16;
            ++np;
            break;
        }
        --i;
        uint64_t ck[4], cl[4];
        occ4_pair(ix, x.k - 1, x.l, ck, cl, fetches);
        const uint64_t kk0 = ix.C[0] + ck[0] + 1, ll0 = ix.C[0] + cl[0];
        const uint64_t kk1 = ix.C[1] + ck[1] + 1, ll1 = ix.C[1] + cl[1];
        const uint64_t kk2 = ix.C[2] + ck[2] + 1, ll2 = ix.C[2] + cl[2];
        const uint64_t kk3 = ix.C[3] + ck[3] + 1, ll3 = ix.C[3] + cl[3];
        uint64_t occ = x.l - x.k + 1;
        int allow_diff = 1, allow_M = 1;
        if (i > 0) {
            uint64_t wa = S->W[i - 1], wb = S->W[i];
            int ba = (int)(wa >> 48), bb = (int)(wb >> 48);
            if (ba > m - 1) allow_diff = 0;
            else if (ba == m - 1 && bb == m - 1 && (wa & kW48) == (wb & kW48)) allow_M = 0;
            int ii = i - (c.len - c.seed_len_r);
            if (c.use_seed && ii > 0) {
                int m_seed = O.max_seed_diff - diffs;
                uint64_t sa = S->SW[ii - 1], sb = S->SW[ii];
                int sba = (int)(sa >> 48), sbb = (int)(sb >> 48);
                if (sba > m_seed - 1) allow_diff = 0;
                else if (sba == m_seed - 1 && sbb == m_seed - 1 && (sa & kW48) == (sb & kW48)) allow_M = 0;
            }
        }
        int gaps = x.n_gapo + x.n_gape;
        int tmp = (O.mode & kModeLoggap) ? (gaps ? (31 - __clz(gaps)) : 0) / 2 + 1 : gaps;
        if (allow_diff && i >= O.indel_end_skip + tmp && c.len - i >= O.indel_end_skip + tmp) {
            if (x.state == kStM) {
                if (x.n_gapo < O.max_gapo) {
                    WPUSH(1, b + O.s_gapo, x.k, x.l, i, x.n_mm, x.n_gapo + 1, x.n_gape, x.n_ins + 1, kStI, 1);
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        uint64_t kk = sel4(cc, kk0, kk1, kk2, kk3), ll = sel4(cc, ll0, ll1, ll2, ll3);
                        if (!err && kk <= ll)
                            WPUSH(1, b + O.s_gapo, kk, ll, i + 1, x.n_mm, x.n_gapo + 1, x.n_gape, x.n_ins, kStD, 1);
                    }
                }
            } else if (x.state == kStI) {
                if (x.n_gape < O.max_gape)
                    WPUSH(2, b + O.s_gape, x.k, x.l, i, x.n_mm, x.n_gapo, x.n_gape + 1, x.n_ins + 1, kStI, 1);
            } else if (x.state == kStD) {
                if (x.n_gape < O.max_gape && (gaps < c.max_diff || occ < (uint64_t)(int64_t)O.max_del_occ)) {
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) {
                        uint64_t kk = sel4(cc, kk0, kk1, kk2, kk3), ll = sel4(cc, ll0, ll1, ll2, ll3);
                        if (!err && kk <= ll)
                            WPUSH(2, b + O.s_gape, kk, ll, i + 1, x.n_mm, x.n_gapo, x.n_gape + 1, x.n_ins, kStD, 1);
                    }
                }
            }
        }
        const int base = S->q[i];
        bool exact = false;
        uint64_t ek = 0, el = 0;
        if (err) {
        } else if (allow_diff && allow_M) {
#pragma unroll
            for (int j = 1; j <= 4; ++j) {
                int cc = (base + j) & 3;
                int mm = j != 4 || base > 3;
                uint64_t kk = sel4(cc, kk0, kk1, kk2, kk3), ll = sel4(cc, ll0, ll1, ll2, ll3);
                if (!err && kk <= ll) {
                    if (!mm) { exact = true; ek = kk; el = ll; }
                    else WPUSH(0, b + O.s_mm, kk, ll, i, x.n_mm + 1, x.n_gapo, x.n_gape, x.n_ins, kStM, 1);
                }
            }
        } else if (base < 4) {
            uint64_t kk = sel4(base, kk0, kk1, kk2, kk3), ll = sel4(base, ll0, ll1, ll2, ll3);
            if (kk <= ll) { exact = true; ek = kk; el = ll; }
        }
        const uint32_t fpop = (fetches - f_pop) << 16;
        if (err) {   // the read ends at this pop with BWTGAP_ERR_SCORE
            S->meta[lane][np] = fpop; ++np; endc = 3; break;
        }
        if (exact) hx = 1;
        S->meta[lane][np] = npu | (hx << 8) | fpop;
        ++np;
        if (!exact) { endc = 0; break; }
        x.k = ek; x.l = el; x.i = i; x.isdiff = 0; x.state = kStM;
        // room for one more pop: at most 9 pushes, all possibly in one list
        if (np == kWR || nl0 + 9 > kWL || nl1 + 9 > kWL || nl2 + 9 > kWL) { endc = 2; S->lane_x[lane] = wpack(x); break; }
    }
#undef WPUSH
    S->lane_np[lane] = np;
    S->lane_end[lane] = endc;
    S->lane_nl[lane][0] = (uint32_t)nl0;
    S->lane_nl[lane][1] = (uint32_t)nl1;
    S->lane_nl[lane][2] = (uint32_t)nl2;
}

// the warp's chunk allocator (warp-uniform state; every lane holds the same copy)
struct WAlloc {
    int32_t *free_ids;
    int base, cap, bump, free_top;
    // `need` chunk ids into out[0..need), lane-parallel; false if the arena is exhausted
    __device__ __forceinline__ bool alloc_n(int need, int32_t *out, int lane)
    {
        bool ok = true;
        for (int t0 = 0; t0 < need; t0 += 32) {
            int t = t0 + lane;
            if (t < need) {
                int id;
                if (t < free_top) id = free_ids[free_top - 1 - t];
                else id = bump + (t - free_top) < cap ? base + bump + (t - free_top) : -1;
                out[t] = id;
            }
        }
        int from_free = need < free_top ? need : free_top;
        if (bump + (need - from_free) > cap) ok = false;
        else { free_top -= from_free; bump += need - from_free; }
        __syncwarp();
        return ok;
    }
    __device__ __forceinline__ void release(int id, int lane)
    {
        if (lane == 0) free_ids[free_top] = id;
        ++free_top;
    }
};

template <bool TRACE>
__device__ void warp_read(const WArgs &a, int pos, int wid, WarpSmem *S, int lane)
{
    const unsigned FULL = 0xffffffffu;
    const int r = a.list[pos];
    const int64_t s0 = a.off[r];
    const int len = (int)(a.off[r + 1] - s0);
    const BatchOpt O = a.bopt[a.bidx[r]];
    const int max_diff0 = a.maxdiff[r];
    const IndexView &ix = a.ix;
    for (int t = lane; t < len; t += 32) S->q[t] = a.query[s0 + t];
    for (int t = lane; t < kWMaxB; t += 32) { S->top_chunk[t] = -1; S->n_in[t] = 0; S->top_cnt[t] = 0; }
    if (lane < kWMaxB / 32) S->mask[lane] = 0;
    __syncwarp();
    uint32_t fetches = 0;   // index blocks read by this lane (chains include discarded speculation)
    const bool use_seed = len > O.seed_len;
    if (lane == 0) {
        cal_width(ix, len, S->q, S->W, fetches);
        if (use_seed) cal_width(ix, O.seed_len, S->q + (len - O.seed_len), S->SW, fetches);
    }
    __syncwarp();
    uint32_t f_alg = __shfl_sync(FULL, fetches, 0);   // algorithmic count: widths, then replayed chains
    uint4 *chunks = a.chunks;
    WAlloc A;
    A.free_ids = a.free_ids + (size_t)wid * a.arena_chunks;
    A.base = wid * a.arena_chunks; A.cap = a.arena_chunks; A.bump = 0; A.free_top = 0;
    uint4 *stage_lane = a.stage + (size_t)wid * 3 * 32 * kWL + (size_t)lane * kWL;   // list L at + L * 32 * kWL
    uint4 *prec_w = a.prec + (size_t)wid * 32 * kWR;
    // the staging list of each push kind: kinds whose target buckets coincide share a list, so the
    // bucket keeps the push order
    int tl[3];
    tl[0] = 0;
    tl[1] = O.s_gapo == O.s_mm ? 0 : 1;
    tl[2] = O.s_gape == O.s_mm ? 0 : (O.s_gape == O.s_gapo ? tl[1] : 2);
    const int lst_pen[3] = {O.s_mm, tl[1] == 1 ? O.s_gapo : -1, tl[2] == 2 ? O.s_gape : -1};
    uint64_t *aln = a.aln + (size_t)wid * a.aln_cap * 3;

    WCtx c;
    c.len = len; c.max_diff0 = max_diff0; c.max_diff = max_diff0; c.use_seed = use_seed;
    c.seed_len_r = len > O.seed_len ? O.seed_len : 0x7fffffff;
    c.gape = (O.mode & kModeGape) != 0; c.nonstop = (O.mode & kModeNonstop) != 0;
    const int n_stacks = O.n_stacks;
    int best_score = (max_diff0 + 1) * O.s_mm + (O.max_gapo + 1) * O.s_gapo + (O.max_gape + 1) * O.s_gape;
    int best_cnt = 0, n_aln = 0, ret = 0, n_entries = 0, peak = 0;
    uint64_t pops = 0, trace = kTraceInit;
    unsigned long long d_waves = 0, d_lanes = 0, d_cons = 0, d_cont = 0, d_hz = 0, d_chainpops = 0;
    long long c_chain = 0, c_replay = 0, c_commit = 0, c_load = 0, t_mark = 0;
    const bool dbg = a.dbg != nullptr;

    int n_amb = 0;
    for (int j = 0; j < len; ++j) n_amb += S->q[j] > 3;
    if (n_amb > c.max_diff) goto publish;

    {
        // the root is the pending entry of the first wave
        bool pend = true;
        int pend_b = 0;
        WEnt px;
        px.k = 0; px.l = ix.seq_len; px.i = len; px.isdiff = 0; px.n_mm = px.n_gapo = px.n_gape = px.n_ins = 0;
        px.state = kStM;
        if (n_stacks <= 0) { ret = kErrScore; goto publish; }
        n_entries = 1; peak = 1;
        for (;;) {
            if (n_entries == 0) break;
            if (n_entries > O.max_entries) break;
            // the bucket of the next pop
            int b;
            if (pend) b = pend_b;
            else {
                b = kWMaxB;
                for (int w = 0; w < kWMaxB / 32; ++w)
                    if (S->mask[w]) { b = w * 32 + __ffs(S->mask[w]) - 1; break; }
            }
            if (b >= kWMaxB || (!pend && S->n_in[b] <= 0)) { ret = kErrStack; break; }   // inconsistent: re-run elsewhere
            const uint32_t binfo = (uint32_t)b << 21;
            if (dbg) t_mark = clock64();
            const int navail = (pend ? 1 : 0) + S->n_in[b];
            const int Wn = navail < 32 ? navail : 32;
            // load the wave's entries: lane 0 the pending child (if any), then the bucket from the top
            WEnt x;
            x.k = 0; x.l = 0; x.i = 0; x.isdiff = 0; x.n_mm = x.n_gapo = x.n_gape = x.n_ins = 0; x.state = 0;
            if (lane < Wn) {
                if (pend && lane == 0) x = px;
                else {
                    int d = lane - (pend ? 1 : 0);
                    int tc = S->top_chunk[b], cnt = S->top_cnt[b];
                    uint4 v = make_uint4(0, 0, 0, 0);
                    if (tc >= 0 && d < cnt) v = chunks[(size_t)tc * kWCH + (cnt - 1 - d)];
                    else if (tc >= 0) {
                        int pc = a.chunk_prev[tc];
                        if (pc >= 0 && d - cnt < kWCH) v = chunks[(size_t)pc * kWCH + (kWCH - 1 - (d - cnt))];
                    }
                    x = wunpack(v);
                }
            }
            // early stop (the same for the whole bucket until a hit): the sequential search pops one entry
            if (!c.nonstop && (binfo >> 21) > (uint32_t)(best_score + O.s_mm)) {
                --n_entries;
                ++pops;
                if (TRACE) {
                    WEnt y;
                    y.k = __shfl_sync(FULL, x.k, 0); y.l = __shfl_sync(FULL, x.l, 0);
                    y.i = __shfl_sync(FULL, x.i, 0); y.isdiff = __shfl_sync(FULL, x.isdiff, 0);
                    y.n_mm = __shfl_sync(FULL, x.n_mm, 0); y.n_gapo = __shfl_sync(FULL, x.n_gapo, 0);
                    y.n_gape = __shfl_sync(FULL, x.n_gape, 0); y.n_ins = __shfl_sync(FULL, x.n_ins, 0);
                    y.state = __shfl_sync(FULL, x.state, 0);
                    uint64_t h = trace;
                    h = trace_mix(h, binfo | (uint32_t)y.i);
                    h = trace_mix(h, y.k);
                    h = trace_mix(h, y.l);
                    h = trace_mix(h, (uint64_t)((uint32_t)y.n_mm | (uint32_t)y.n_gapo << 8 | (uint32_t)y.n_gape << 16
                                                | (uint32_t)y.state << 24));
                    int n_del = y.n_gapo + y.n_gape - y.n_ins;
                    h = trace_mix(h, (uint64_t)(y.n_ins & 0xffff) | (uint64_t)(n_del & 0xffff) << 16);
                    h = trace_mix(h, (uint64_t)(uint32_t)(y.isdiff ? y.i : 0));
                    h = trace_mix(h, (uint64_t)(uint32_t)n_entries);
                    trace = h;
                }
                break;
            }
            // speculative chains
            if (dbg) { long long t = clock64(); c_load += t - t_mark; t_mark = t; }
            if (lane < Wn) lane_chain<TRACE>(ix, O, c, S, lane, x, b, fetches, stage_lane, tl, prec_w + (size_t)lane * kWR);
            __syncwarp();
            if (dbg) {
                long long t = clock64(); c_chain += t - t_mark; t_mark = t;
                ++d_waves; d_lanes += Wn;
                for (int j = 0; j < Wn; ++j) d_chainpops += S->lane_np[j];
            }
            // replay in sequential order. Without the trace hash, the lanes before the first lane that
            // stops the replay (a hit, an error, an unfinished chain, or the max_entries cut-off inside its
            // chain) are replayed at once from prefix sums; that lane, and in trace mode every lane, one pop
            // at a time.
            int consumed = 0;          // lanes whose entries are consumed
            bool stop = false, search_end = false, new_pend = false;
            int j_first = 0;
            if (!TRACE) {
                const int npl = lane < Wn ? S->lane_np[lane] : 0;
                const int endl = lane < Wn ? S->lane_end[lane] : 0;
                int pre = 0, mpre = 0, pmax = 0;
                uint32_t fsum = 0;
                for (int t = 0; t < npl; ++t) {
                    const uint32_t meta = S->meta[lane][t];
                    if (pre > mpre) mpre = pre;          // n_entries before pop t, relative to the chain start
                    pre += (int)(meta & 0xff) + (int)((meta >> 8) & 1) - 1;
                    if (pre > pmax) pmax = pre;
                    fsum += meta >> 16;
                }
                int incl = pre;
                for (int o = 1; o < 32; o <<= 1) {
                    int v = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += v;
                }
                const int nstart = n_entries + incl - pre;
                const bool cross = lane < Wn && nstart + mpre > O.max_entries;
                const unsigned bal = __ballot_sync(FULL, lane < Wn && (cross || endl != 0));
                const int sstar = bal ? __ffs(bal) - 1 : Wn;
                const bool take = lane < sstar;
                pops += (uint64_t)__reduce_add_sync(FULL, take ? (unsigned)npl : 0u);
                n_entries += (int)__reduce_add_sync(FULL, take ? (unsigned)pre : 0u);
                f_alg += __reduce_add_sync(FULL, take ? fsum : 0u);
                const int pk = (int)__reduce_max_sync(FULL, take ? (unsigned)(nstart + pmax) : 0u);
                if (pk > peak) peak = pk;
                consumed = sstar;
                j_first = sstar;
            }
            for (int j = j_first; j < Wn && !stop && (TRACE || j == j_first); ++j) {
                const int np = S->lane_np[j], endc = S->lane_end[j];
                for (int t = 0; t < np; ++t) {
                    if (n_entries > O.max_entries) { search_end = true; stop = true; break; }
                    --n_entries;
                    ++pops;
                    const uint32_t meta = S->meta[j][t];
                    f_alg += meta >> 16;
                    if (TRACE) {
                        WEnt y = wunpack(prec_w[(size_t)j * kWR + t]);
                        uint64_t h = trace;
                        h = trace_mix(h, binfo | (uint32_t)y.i);
                        h = trace_mix(h, y.k);
                        h = trace_mix(h, y.l);
                        h = trace_mix(h, (uint64_t)((uint32_t)y.n_mm | (uint32_t)y.n_gapo << 8
                                                    | (uint32_t)y.n_gape << 16 | (uint32_t)y.state << 24));
                        int n_del = y.n_gapo + y.n_gape - y.n_ins;
                        h = trace_mix(h, (uint64_t)(y.n_ins & 0xffff) | (uint64_t)(n_del & 0xffff) << 16);
                        h = trace_mix(h, (uint64_t)(uint32_t)(y.isdiff ? y.i : 0));
                        h = trace_mix(h, (uint64_t)(uint32_t)n_entries);
                        trace = h;
                    }
                    if (t == np - 1 && endc == 3) { ret = kErrScore; search_end = true; stop = true; break; }
                    if (t == np - 1 && endc == 1) {
                        // the hit, as bwt_match_gap handles it
                        consumed = j + 1;
                        stop = true;
                        WEnt e = wunpack(S->hz[j]);
                        uint64_t k = S->hk[j], l = S->hl[j];
                        int sc = e.n_mm * O.s_mm + e.n_gapo * O.s_gapo + e.n_gape * O.s_gape;
                        int diffs = e.n_mm + e.n_gapo + (c.gape ? e.n_gape : 0);
                        if (n_aln == 0) {
                            best_score = sc;
                            if (!c.nonstop) c.max_diff = diffs + 1 > max_diff0 ? max_diff0 : diffs + 1;
                        }
                        if (sc == best_score) best_cnt = (int)(uint32_t)((uint64_t)(int64_t)best_cnt + (l - k + 1));
                        else if (best_cnt > O.max_top2) { search_end = true; break; }
                        bool add = true;
                        if (e.n_gapo)
                            for (int q = 0; q < n_aln; ++q)
                                if (aln[3 * q + 1] == k && aln[3 * q + 2] == l) { add = false; break; }
                        if (add) {
                            int ldp = e.isdiff ? e.i : 0;
                            uint64_t xx = (uint64_t)(int64_t)(int)(l - k + 1);
                            int jb = 0;
                            for (int t0 = 0; t0 < ldp; t0 += 32) {
                                int tt = t0 + lane;
                                uint64_t v = tt < ldp ? S->W[tt] : 0, wv = v & kW48;
                                bool eq = tt < ldp && wv == xx, gt = tt < ldp && wv > xx;
                                unsigned bal = __ballot_sync(FULL, eq);
                                int rank = __popc(bal & ((1u << lane) - 1));
                                if (gt) S->W[tt] = (v & ~kW48) | (wv - xx);
                                if (eq) S->W[tt] = (1ull << 48) | ((ix.seq_len - (uint64_t)(jb + rank + 1)) & kW48);
                                jb += __popc(bal);
                            }
                            __syncwarp();
                            if (n_aln == a.aln_cap) { ret = kErrAln; search_end = true; break; }
                            if (lane == 0) {
                                int n_del = e.n_gapo + e.n_gape - e.n_ins;
                                aln[3 * n_aln] = (uint64_t)(e.n_mm & 0xff) | (uint64_t)(e.n_gapo & 0xff) << 8
                                               | (uint64_t)(e.n_gape & 0xff) << 16 | (uint64_t)(sc & 0xfffff) << 24
                                               | (uint64_t)(e.n_ins & 0x3ff) << 44 | (uint64_t)(n_del & 0x3ff) << 54;
                                aln[3 * n_aln + 1] = k;
                                aln[3 * n_aln + 2] = l;
                            }
                            __syncwarp();
                            ++n_aln;
                        }
                        break;
                    }
                    n_entries += (int)(meta & 0xff) + (int)((meta >> 8) & 1);
                    if (n_entries > peak) peak = n_entries;
                }
                if (stop) break;
                consumed = j + 1;
                if (endc == 2) { new_pend = true; stop = true; }
            }
            if (dbg) {
                long long t = clock64(); c_replay += t - t_mark; t_mark = t;
                d_cons += consumed; d_cont += new_pend ? 1 : 0;
                if (consumed > 0 && S->lane_end[consumed - 1] == 1) ++d_hz;
            }
            if (search_end) break;
            // take the consumed entries off bucket b (lane 0 of the wave may have been the pending child)
            int C = consumed - (pend ? 1 : 0);
            if (C > 0) {
                int tc = S->top_chunk[b], cnt = S->top_cnt[b];
                if (tc < 0) { ret = kErrStack; break; }
                __syncwarp();
                if (C < cnt) {
                    if (lane == 0) S->top_cnt[b] = (uint16_t)(cnt - C);
                } else {
                    int pc = a.chunk_prev[tc];
                    A.release(tc, lane);
                    int rest = C - cnt;    // entries taken from the previous chunk
                    if (pc >= 0 && rest == kWCH) { int pp = a.chunk_prev[pc]; A.release(pc, lane); pc = pp; rest = 0; }
                    if (lane == 0) {
                        S->top_chunk[b] = pc;
                        S->top_cnt[b] = (uint16_t)(pc >= 0 ? kWCH - rest : 0);
                    }
                }
                if (lane == 0) {
                    S->n_in[b] -= C;
                    if (S->n_in[b] == 0) S->mask[b >> 5] &= ~(1u << (b & 31));
                }
                __syncwarp();
            }
            pend = false;
            if (new_pend) {
                pend = true;
                pend_b = b;
                px = wunpack(S->lane_x[consumed - 1]);
            }
            // commit the pushes of the consumed lanes, list by list (one list per target bucket), in replay
            // order: lane order, then the order the lane staged them
            bool fail = false;
            for (int L = 0; L < 3 && !fail; ++L) {
                if (lst_pen[L] < 0) continue;
                const int X = b + lst_pen[L];
                int cntX = lane < consumed ? (int)S->lane_nl[lane][L] : 0;
                int incl = cntX;
                for (int o = 1; o < 32; o <<= 1) {
                    int v = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += v;
                }
                const int T = __shfl_sync(FULL, incl, 31);
                if (T == 0) continue;
                if (X >= n_stacks || X >= kWMaxB) { ret = kErrScore; fail = true; break; }
                const int c0 = S->top_chunk[X], cnt0 = c0 >= 0 ? S->top_cnt[X] : 0;
                const int need = (cnt0 + T + kWCH - 1) / kWCH - (c0 >= 0 ? 1 : 0);
                if (need > kWNewC || !A.alloc_n(need, S->newc, lane)) { ret = kErrStack; fail = true; break; }
                // chain the new chunks on top of c0
                for (int t = lane; t < need; t += 32) a.chunk_prev[S->newc[t]] = t == 0 ? c0 : S->newc[t - 1];
                // copy: output position p (0..T) comes from the lane j with incl[j-1] <= p < incl[j]
                S->incl[lane] = incl;
                __syncwarp();
                const uint4 *stw = a.stage + (size_t)wid * 3 * 32 * kWL + (size_t)L * 32 * kWL;
                for (int p0 = 0; p0 < T; p0 += 32) {
                    const int p = p0 + lane;
                    if (p < T) {
                        int lo = 0, hi = 31;          // first lane whose inclusive count exceeds p
                        while (lo < hi) {
                            int mid = (lo + hi) >> 1;
                            if (S->incl[mid] > p) hi = mid; else lo = mid + 1;
                        }
                        const int before = lo ? S->incl[lo - 1] : 0;
                        const int g = cnt0 + p;
                        const int ci = g / kWCH;
                        const int chunk = c0 >= 0 ? (ci == 0 ? c0 : S->newc[ci - 1]) : S->newc[ci];
                        chunks[(size_t)chunk * kWCH + (g % kWCH)] = stw[(size_t)lo * kWL + (p - before)];
                    }
                }
                __syncwarp();
                if (lane == 0) {
                    int last = cnt0 + T - 1;
                    int ci = last / kWCH;
                    S->top_chunk[X] = c0 >= 0 ? (ci == 0 ? c0 : S->newc[ci - 1]) : S->newc[ci];
                    S->top_cnt[X] = (uint16_t)(last % kWCH + 1);
                    S->n_in[X] += T;
                    S->mask[X >> 5] |= 1u << (X & 31);
                }
                __syncwarp();
            }
            if (dbg) { long long t = clock64(); c_commit += t - t_mark; }
            if (fail) break;
        }
        if (ret == 0) ret = n_aln;
    }
publish:
    if (ret > 0) {
        unsigned long long o = 0;
        if (lane == 0) o = atomicAdd(a.rec_top, (unsigned long long)ret);
        o = __shfl_sync(FULL, o, 0);
        if ((int64_t)(o + ret) > a.rec_cap) ret = kErrAln;
        else {
            for (int j = lane; j < 3 * ret; j += 32) a.out_rec[o * 3 + j] = aln[j];
            if (lane == 0) a.out_off[r] = (int64_t)o;
        }
    }
    if (dbg && lane == 0) {
        atomicAdd(a.dbg + kDbgReads, 1ull);
        atomicAdd(a.dbg + kDbgWaves, d_waves);
        atomicAdd(a.dbg + kDbgLanes, d_lanes);
        atomicAdd(a.dbg + kDbgConsumed, d_cons);
        atomicAdd(a.dbg + kDbgPops, (unsigned long long)pops);
        atomicAdd(a.dbg + kDbgCont, d_cont);
        atomicAdd(a.dbg + kDbgHazard, d_hz);
        atomicAdd(a.dbg + kDbgCycChain, (unsigned long long)c_chain);
        atomicAdd(a.dbg + kDbgCycReplay, (unsigned long long)c_replay);
        atomicAdd(a.dbg + kDbgCycCommit, (unsigned long long)c_commit);
        atomicAdd(a.dbg + kDbgCycLoad, (unsigned long long)c_load);
        atomicAdd(a.dbg + kDbgChainPops, d_chainpops);
    }
    if (lane == 0) {
        if (ret == kErrStack || ret == kErrAln) a.ovf[atomicAdd(a.ovf_n, 1)] = r;
        a.out_n[r] = ret;
        a.out_pops[r] = pops;
        a.out_trace[r] = TRACE ? trace : 0;
        a.out_peak[r] = peak;
        a.out_fetch[r] = f_alg;
        a.out_tier[r] = (int8_t)a.tier;
    }
    __syncwarp();
}

template <bool TRACE>
__global__ void __launch_bounds__(32) warp_kernel(const __grid_constant__ WArgs a)
{
    extern __shared__ __align__(16) unsigned char wsm_raw[];
    WarpSmem *S = (WarpSmem *)wsm_raw;
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x;
    if (wid >= a.n_warps) return;
    for (;;) {
        int pos = 0;
        if (lane == 0) pos = atomicAdd(a.claim, 1);
        pos = __shfl_sync(0xffffffffu, pos, 0);
        if (pos >= a.n) break;
        warp_read<TRACE>(a, pos, wid, S, lane);
    }
}

}  // namespace galn
