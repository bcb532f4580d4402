// galn_warp.cuh -- the heavy-read tier: one warp per read, many stack entries expanded at once.
//
// Why this is exact. With positive penalties (s_mm, s_gapo, s_gape > 0) every child of an entry popped from
// score bucket b goes to a bucket above b, except the exact-match child, which has score b and is pushed
// last, so it is the very next pop (src/bwtgap_hd.h:457-470 push order). Bucket b therefore receives no
// entry while it is being popped: its pops are the entries e_m, e_{m-1}, ..., e_1 (LIFO), each followed
// by its chain of exact-match children. Between two hits the expansion of a chain depends only on its
// first entry, the width arrays and max_diff, none of which change without a hit; so the chains of the
// top entries of bucket b can be expanded at the same time, in any order and on any lane.
//
// One wave takes up to kWE entries from the top of bucket b (entry 0 may be a pending exact child left by
// the previous wave). The warp runs in steps: in each step every busy lane expands one pop of its chain,
// and every idle lane takes the next entry not yet handed out (in entry order), so lanes stay busy however
// uneven the chains are. A lane stages the pushes of each pop (in the order bwt_match_gap pushes them) in
// global memory, one list per distinct target bucket (b+s_mm, b+s_gapo, b+s_gape), and 2 bytes of per-pop
// data in the warp's side area; when a chain ends it writes the entry's record (its lane, pops, staged segments
// and prefix sums). A chain that reaches a hit, a score past n_stacks, or the end of its lane's space
// (a "stop") ends the hand-out after its entry; entries past it are dropped.
//
// Then the warp replays the entries in order exactly as the sequential search would pop them: the
// max_entries test before each pop, n_entries after each pop and push, the pop count, the trace hash, the
// first hit (handled sequentially: best_score, max_diff, -R, gapped-hit de-duplication, gap_shadow, the
// record). Without the trace hash the entries before the first stop are replayed at once from prefix
// sums; that entry (and, in trace mode, every entry) one pop at a time. The pushes of the replayed entries
// are committed to their buckets in replay order (per bucket: entry order, then pop order), so every
// bucket is the same LIFO as in the sequential search.
//
// Storage: each bucket is a chain of 64-entry chunks in the warp's arena (global memory), with its top
// chunk, fill and entry count in shared memory. Widths, the query, the wave's entries and records are in
// shared memory; the per-pop data, staged pushes (and, in trace mode, popped entries) in per-warp global
// areas. Reads the tier cannot take (length > 256, n_stacks > 128, a penalty <= 0, 32-byte
// entries) or that outgrow the arena or the record buffer go to the thread tiers (the host routes them).
#pragma once

#include "galn_internal.h"
#include "galn_search.cuh"

namespace galn {

constexpr int kWMaxB = kWarpMaxStacks;   // buckets
constexpr int kWMaxLen = kWarpMaxLen;    // read length
constexpr int kWE = 192;         // entries per wave
constexpr int kEPL = kWE / 32;   // entries per lane in the replay and commit scans (lane j: entries kEPL*j ..)
static_assert(kWE % 32 == 0 && kWMaxB % 32 == 0, "wave and bucket layouts");
constexpr int kWP = 48;          // pops per lane per wave
constexpr int kWL = 128;         // staged pushes per lane and target list per wave
static_assert(kWL <= 255, "a staged segment's start and count are 8-bit fields");
constexpr int kWCH = kWarpChunk;  // entries per chunk
constexpr int kWNewC = (kWCH + 32 * kWL) / kWCH + 2;   // chunks one commit may allocate
constexpr int kWGrabPops = 6;    // an idle lane takes an entry only with room for this many pops
constexpr int kWChain = kWE / kWCH + 2;   // chunks of the current bucket kept walked
constexpr int kFC = 64;          // free chunk ids kept in shared memory

constexpr int kWDbgN = 15;       // optional counters per read (the kDbg* list below)

struct WarpSmem {
    int32_t top_chunk[kWMaxB];
    int32_t n_in[kWMaxB];
    uint16_t top_cnt[kWMaxB];
    uint32_t mask[kWMaxB / 32];
    uint64_t W[kWMaxLen + 1];
    uint64_t SW[kWMaxLen + 1];
    uint8_t q[kWMaxLen];
    uint4 ent[kWE];                   // the wave's entries, in pop order
    uint32_t e_info[kWE];             // per entry: lane (bits 0-7), first pop (8-15), pops (16-23), end code (24-31)
    uint16_t e_seg[3][kWE];           // per entry and list: first staged push (bits 0-7), count (8-15); both <= kWL
    uint32_t e_a[kWE];                // per entry: net change of n_entries (signed, bits 0-15), its highest value before a pop (16-31)
    uint32_t e_b[kWE];                // per entry: highest value after a pop (bits 0-15), index blocks read (16-31)
    int32_t newc[kWNewC];             // chunks allocated for one commit
    int32_t wch[kWChain];             // the current bucket's chunks from its top, as far as walked
    int32_t fcache[kFC];              // the top of the warp's free-chunk stack
    BatchOpt O;                       // the read's batch options (read from here, not held in registers)
    unsigned long long dv[kWDbgN];    // optional counters of this read (profiling runs)
    long long t_mark, t_read;
};

// Per-warp data that is written often but read rarely (at hits, pending children and the one entry a wave
// replays pop by pop), kept in global memory to leave shared memory for more resident warps.
struct WSide {
    uint4 hz[32];                     // hazard entry of each lane
    uint4 lane_x[32];                 // pending exact child of a lane that stopped mid-chain
    uint64_t hk[32], hl[32];          // the hazard's interval after the exact tail
    // per pop of each lane: pushes (bits 0-3, the fused exact child not counted), has an exact child
    // (bit 4), index blocks read (bits 5-15). Pop-major: the lanes of one step write neighbouring halfwords,
    // so a step's writes fill a few sectors instead of touching one sector per lane.
    uint16_t meta[kWP][32];
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
    uint4 *prec;              // n_warps * 32 lanes * kWP popped entries (trace mode)
    WSide *side;              // n_warps
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
    // Warps 0..n_big-1 have arenas of big_chunks chunks (room for the max_entries cut-off); the others
    // arena_chunks. A read that outgrows a small arena is queued in ovq (its tail at q_ctl[1]) for the big
    // warps, which take queued reads before new ones (q_ctl: 0 head, 1 tail, 2 small warps finished,
    // 3 set when a big warp gave up waiting; the host then re-runs every queued read).
    int n_big, big_chunks;
    int32_t *ovq;
    int32_t *q_ctl;
    uint64_t q_wait_ns;       // a big warp gives up waiting for queued work after this long
    unsigned long long *dbg;  // optional counters (kWDbg entries), or NULL
};

// optional counters of the warp tier (per launch, summed over warps)
enum { kDbgReads, kDbgWaves, kDbgLanes, kDbgConsumed, kDbgPops, kDbgCont, kDbgHazard, kDbgCycChain,
       kDbgCycReplay, kDbgCycCommit, kDbgCycLoad, kDbgChainPops, kDbgCycRead, kDbgSteps, kDbgCycReadMax, kWDbg };
static_assert(kWDbg == kWDbgN, "counter list");

// profiling helpers: lane 0 keeps the read's counters in shared memory
#define WDBG_ADD(K, V) do { if (dbg && lane == 0) S->dv[K] += (unsigned long long)(V); } while (0)
#define WDBG_LAP(K) do { if (dbg && lane == 0) { long long t_ = clock64(); S->dv[K] += (unsigned long long)(t_ - S->t_mark); S->t_mark = t_; } } while (0)

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

// one asynchronous 16-byte copy from global to shared memory, through L2 (cp.async.cg: staged pushes were
// written by other lanes of the warp), and the wait for all of the thread's copies
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(s), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

struct WCtx {
    int len, max_diff, max_diff0, use_seed, seed_len_r;
    bool gape, nonstop;
};

// The exact walk of a pop with no difference left (bwt_match_exact_alt, src/bwtgap_hd.h:195-211), kept
// across steps: one LF step per warp step, so that it shares the step's single index fetch with the other
// lanes' pops instead of stalling the warp for its whole length.
struct WWalk {
    uint64_t k, l;
    int i;                 // bases left to match (positions i-1 .. 0)
    uint32_t f;            // index blocks read by the walk so far
    bool on;
};

// One step of a lane's chain: a pop, or one LF step of a pop's exact walk. Returns the chain's end code:
// -2 = the pop's exact walk goes on (no pop finished), -1 = the pop finished and the chain continues with
// its exact child (now in x), 0 = the chain is finished, 1 = hazard (a hit) at this pop, 2 = stopped with
// the exact child pending (no room left in this wave; the child is in D->lane_x), 3 = this pop pushes a
// score >= n_stacks (bwt_match_gap returns BWTGAP_ERR_SCORE there). A finished pop's data goes to
// D->meta[lp][lane] (and to mt); its pushes are appended to this lane's staging lists (st: list L at
// st + L * 32 * kWL; tl: list of each push kind, mismatch, gap open, gap extension); in trace mode the popped
// entry goes to pr[lp].
template <bool TRACE, int ST>
__device__ __forceinline__ int lane_step(const IndexView &ix, const BatchOpt &O, const WCtx &c, WarpSmem *S, WSide *D,
                                         int lane, WEnt &x, WWalk &wk, int b, uint32_t &fetches, uint4 *st, const int tl[3],
                                         uint4 *pr, int &lp, int &nl0, int &nl1, int &nl2, uint32_t &mt)
{
    const size_t lstride = (size_t)32 * kWL;
    bool err = false;
    uint32_t npu = 0;
    int endc = -2;
    bool load = false;           // this step reads Occ at (k1, l1)
    uint64_t k1 = 0, l1 = 0;
    int diffs = 0, m = 0, i = x.i;
    // ---- before the fetch: the tests that need no index data ----
    if (wk.on) {
        if (S->q[wk.i - 1] > 3) { wk.on = false; mt = wk.f << 5; endc = 0; }
        else { load = true; k1 = wk.k - 1; l1 = wk.l; }
    } else {
        if (TRACE) pr[lp] = wpack(x);
        diffs = x.n_mm + x.n_gapo + (c.gape ? x.n_gape : 0);
        m = c.max_diff - diffs;
        if (m < 0 || (i > 0 && m < (int)(S->W[i - 1] >> 48))) {
            mt = 0; endc = 0;
        } else if (i == 0) {
            D->hz[lane] = wpack(x); D->hk[lane] = x.k; D->hl[lane] = x.l;
            mt = 0; endc = 1;
        } else if (m == 0 && (x.state == kStM || c.gape || x.n_gape == O.max_gape)) {
            // bwt_match_exact_alt over positions i-1 .. 0
            if (S->q[i - 1] > 3) { mt = 0; endc = 0; }
            else { wk.on = true; wk.k = x.k; wk.l = x.l; wk.i = i; wk.f = 0; load = true; k1 = x.k - 1; l1 = x.l; }
        } else {
            load = true; k1 = x.k - 1; l1 = x.l;
        }
    }
    // ---- the step's one fetch ----
    uint64_t ck[4], cl[4];
    uint32_t df = 0;
    if (load) {
        const uint32_t f0 = fetches;
        occ4_pair_u<ST>(ix, k1, l1, ck, cl, fetches);
        df = fetches - f0;
    }
    if (load && wk.on) {
        // one LF step of the exact walk
        const int cc = S->q[wk.i - 1];
        const uint64_t kk = ix.C[cc] + sel4(cc, ck[0], ck[1], ck[2], ck[3]) + 1;
        const uint64_t ll = ix.C[cc] + sel4(cc, cl[0], cl[1], cl[2], cl[3]);
        wk.f += df;
        if (kk > ll) { wk.on = false; mt = wk.f << 5; endc = 0; }
        else if (--wk.i == 0) {
            wk.on = false;
            D->hz[lane] = wpack(x); D->hk[lane] = kk; D->hl[lane] = ll;
            mt = wk.f << 5; endc = 1;
        } else { wk.k = kk; wk.l = ll; }
    } else if (load) {
        // the expansion of the pop (src/bwtgap_hd.h:396-470) as nine predicated push slots in the order
        // bwt_match_gap pushes them: the gap child that keeps the interval (insertion open or extension), the
        // four deletion children (open or extension), the mismatches; then the exact child
        --i;
        uint64_t kk[4], ll[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) { kk[q] = ix.C[q] + ck[q] + 1; ll[q] = ix.C[q] + cl[q]; }
        const uint64_t occ = x.l - x.k + 1;
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
        const int gaps = x.n_gapo + x.n_gape;
        const int tmp = (O.mode & kModeLoggap) ? (gaps ? (31 - __clz(gaps)) : 0) / 2 + 1 : gaps;
        const bool indel = allow_diff && i >= O.indel_end_skip + tmp && c.len - i >= O.indel_end_skip + tmp;
        const bool st_m = x.state == kStM, st_i = x.state == kStI;
        const bool open_ok = indel && st_m && x.n_gapo < O.max_gapo;
        const bool ext_i = indel && st_i && x.n_gape < O.max_gape;
        const bool ext_d = indel && x.state == kStD && x.n_gape < O.max_gape
                           && (gaps < c.max_diff || occ < (uint64_t)(int64_t)O.max_del_occ);
        const bool self_ok = open_ok || ext_i;          // insertion: open from M, extension from I
        const bool del_ok = open_ok || ext_d;           // deletions: open from M, extension from D
        const bool mm_ok = allow_diff && allow_M;
        // list and bucket of each slot kind (a gap open from M, an extension otherwise)
        const int g_list = st_m ? tl[1] : tl[2];
        const int g_bkt = b + (st_m ? O.s_gapo : O.s_gape);
        const int m_bkt = b + O.s_mm;
        // the packed words of each slot kind, but for k and l
        const uint64_t gap1 = st_m ? (1ull << 38) : (1ull << 45);    // n_gapo + 1 or n_gape + 1
        const uint64_t w1b = ((uint64_t)(x.n_gapo & 127) << 38) | ((uint64_t)(x.n_gape & 127) << 45)
                           | ((uint64_t)(x.n_ins & 255) << 52);
        const uint64_t w0b = ((uint64_t)(x.n_mm & 127) << 54) | (1ull << 63);
        const uint64_t h0_self = w0b | ((uint64_t)(uint32_t)i << 38) | ((uint64_t)kStI << 61);
        const uint64_t h1_self = w1b + gap1 + (1ull << 52);
        const uint64_t h0_del = w0b | ((uint64_t)(uint32_t)(i + 1) << 38) | ((uint64_t)kStD << 61);
        const uint64_t h1_del = w1b + gap1;
        const uint64_t h0_mm = (w0b + (1ull << 54)) | ((uint64_t)(uint32_t)i << 38) | ((uint64_t)kStM << 61);
        const int base = S->q[i];
        // the children in mismatch order: rk[j], rl[j] = child of base (base + j) & 3 (j = 4: the read's own base,
        // the exact child), a rotation by base & 3 done once with compile-time indices after it
        uint64_t rk[5], rl[5];
        {
            const int r = base & 3;
            uint64_t a0 = kk[0], a1 = kk[1], a2 = kk[2], a3 = kk[3], b0 = ll[0], b1 = ll[1], b2 = ll[2], b3 = ll[3];
            if (r & 1) { uint64_t t = a0; a0 = a1; a1 = a2; a2 = a3; a3 = t; t = b0; b0 = b1; b1 = b2; b2 = b3; b3 = t; }
            if (r & 2) { uint64_t t = a0; a0 = a2; a2 = t; t = a1; a1 = a3; a3 = t; t = b0; b0 = b2; b2 = t; t = b1; b1 = b3; b3 = t; }
            rk[1] = a1; rk[2] = a2; rk[3] = a3; rk[4] = a0;   // a_j = child of base (r + j) & 3
            rl[1] = b1; rl[2] = b2; rl[3] = b3; rl[4] = b0;
            rk[0] = rl[0] = 0;
        }
        // which slots push: bit 0 the kept-interval gap child, bits 1-4 deletions by base, bits 5-8 mismatches
        uint32_t slots = self_ok ? 1u : 0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) if (del_ok && kk[q] <= ll[q]) slots |= 2u << q;
#pragma unroll
        for (int j = 1; j <= 4; ++j) {
            const bool mm = j != 4 || base > 3;
            if (mm_ok && mm && rk[j] <= rl[j]) slots |= 32u << (j - 1);
        }
        // a push at or past n_stacks ends the read (BWTGAP_ERR_SCORE); nothing else of this pop matters then
        err = ((slots & 0x1fu) && g_bkt >= O.n_stacks) || ((slots & 0x1e0u) && m_bkt >= O.n_stacks);
        if (!err) {
            // the gap children (slots 0-4) go to list g_list and the mismatches (slots 5-8) to list 0 (tl[0]),
            // each kind in slot order at consecutive places; when both kinds share list 0 the mismatches follow
            // the gap children, as bwt_match_gap pushes them
            const uint32_t gs = slots & 0x1fu, ms = slots >> 5;
            const int ng = __popc(gs), nm = __popc(ms);
            const int gbase = g_list == 0 ? nl0 : (g_list == 1 ? nl1 : nl2);
            nl0 += g_list == 0 ? ng : 0;
            nl1 += g_list == 1 ? ng : 0;
            nl2 += g_list == 2 ? ng : 0;
            const int gofs = g_list * (int)lstride + gbase, mofs = nl0;
            nl0 += nm;
            npu = (uint32_t)(ng + nm);
#pragma unroll
            for (int t = 0; t < 5; ++t) {
                if (!(gs & (1u << t))) continue;
                const uint64_t w0 = t == 0 ? (x.k & kK38) | h0_self : (kk[t - 1] & kK38) | h0_del;
                const uint64_t w1 = t == 0 ? (x.l & kK38) | h1_self : (ll[t - 1] & kK38) | h1_del;
                st[gofs + __popc(gs & ((1u << t) - 1u))] = make_uint4((uint32_t)w0, (uint32_t)(w0 >> 32), (uint32_t)w1,
                                                                 (uint32_t)(w1 >> 32));
            }
#pragma unroll
            for (int j = 1; j <= 4; ++j) {
                if (!(ms & (1u << (j - 1)))) continue;
                const uint64_t w0 = (rk[j] & kK38) | h0_mm, w1 = (rl[j] & kK38) | w1b;
                st[mofs + __popc(ms & ((1u << (j - 1)) - 1u))] = make_uint4((uint32_t)w0, (uint32_t)(w0 >> 32), (uint32_t)w1,
                                                                      (uint32_t)(w1 >> 32));
            }
        }
        const bool exact = !err && base < 4 && rk[4] <= rl[4];
        if (err) {   // the read ends at this pop with BWTGAP_ERR_SCORE
            mt = df << 5; endc = 3;
        } else {
            mt = npu | (exact ? 16u : 0u) | df << 5;
            endc = exact ? -1 : 0;
            if (exact) { x.k = rk[4]; x.l = rl[4]; x.i = i; x.isdiff = 0; x.state = kStM; }
        }
    }
    if (endc == -2) return endc;
    D->meta[lp][lane] = (uint16_t)mt;
    ++lp;
    // room for one more pop: at most 9 pushes, all possibly in one list
    if (endc == -1 && (lp == kWP || nl0 + 9 > kWL || nl1 + 9 > kWL || nl2 + 9 > kWL)) {
        endc = 2;
        D->lane_x[lane] = wpack(x);
    }
    return endc;
}

// the warp's chunk allocator (warp-uniform state; every lane holds the same copy): a stack of free chunk
// ids whose top kFC entries live in shared memory (fc), the rest in global memory, then fresh chunks
struct WAlloc {
    int32_t *free_ids;
    int32_t *fc;
    int base, cap, bump, g_top, fc_n;
    // `need` chunk ids into out[0..need), lane-parallel; false if the arena is exhausted
    __device__ __forceinline__ bool alloc_n(int need, int32_t *out, int lane)
    {
        const int from_c = need < fc_n ? need : fc_n;
        const int from_g = need - from_c < g_top ? need - from_c : g_top;
        const int from_b = need - from_c - from_g;
        if (bump + from_b > cap) return false;
        for (int t = lane; t < need; t += 32) {
            int id;
            if (t < from_c) id = fc[fc_n - 1 - t];
            else if (t < from_c + from_g) id = free_ids[g_top - 1 - (t - from_c)];
            else id = base + bump + (t - from_c - from_g);
            out[t] = id;
        }
        fc_n -= from_c; g_top -= from_g; bump += from_b;
        __syncwarp();
        return true;
    }
    __device__ __forceinline__ void release(int id, int lane)
    {
        static_assert(kFC == 64, "spill layout");
        if (fc_n == kFC) {   // the cache's lower half to the global stack
            free_ids[g_top + lane] = fc[lane];
            const int v = fc[lane + 32];
            __syncwarp();
            fc[lane] = v;
            g_top += 32; fc_n -= 32;
        }
        if (lane == 0) fc[fc_n] = id;
        ++fc_n;
        __syncwarp();
    }
};

template <bool TRACE>
__device__ __forceinline__ uint64_t trace_pop(uint64_t h, uint32_t binfo, const WEnt &y, int n_entries)
{
    h = trace_mix(h, binfo | (uint32_t)y.i);
    h = trace_mix(h, y.k);
    h = trace_mix(h, y.l);
    h = trace_mix(h, (uint64_t)((uint32_t)y.n_mm | (uint32_t)y.n_gapo << 8 | (uint32_t)y.n_gape << 16
                                | (uint32_t)y.state << 24));
    int n_del = y.n_gapo + y.n_gape - y.n_ins;
    h = trace_mix(h, (uint64_t)(y.n_ins & 0xffff) | (uint64_t)(n_del & 0xffff) << 16);
    h = trace_mix(h, (uint64_t)(uint32_t)(y.isdiff ? y.i : 0));
    h = trace_mix(h, (uint64_t)(uint32_t)n_entries);
    return h;
}

template <bool TRACE, int ST>
__device__ void warp_read(const WArgs &a, int r, int wid, WarpSmem *S, int lane)
{
    const unsigned FULL = 0xffffffffu;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int64_t s0 = a.off[r];
    const int len = (int)(a.off[r + 1] - s0);
    if (lane == 0) S->O = a.bopt[a.bidx[r]];
    __syncwarp();
    const BatchOpt &O = S->O;
    const int max_diff0 = a.maxdiff[r];
    const IndexView &ix = a.ix;
    for (int t = lane; t < len; t += 32) S->q[t] = a.query[s0 + t];
    for (int t = lane; t < kWMaxB; t += 32) { S->top_chunk[t] = -1; S->n_in[t] = 0; S->top_cnt[t] = 0; }
    if (lane < kWMaxB / 32) S->mask[lane] = 0;
    __syncwarp();
    uint32_t fetches = 0;   // index blocks read by this lane (chains include discarded speculation)
    const bool use_seed = len > O.seed_len;
    if (lane == 0) {
        cal_width<ST>(ix, len, S->q, S->W, fetches);
        if (use_seed) cal_width<ST>(ix, O.seed_len, S->q + (len - O.seed_len), S->SW, fetches);
    }
    __syncwarp();
    uint32_t f_alg = __shfl_sync(FULL, fetches, 0);   // algorithmic count: widths, then replayed chains
    uint4 *chunks = a.chunks;
    WAlloc A;
    {
        const bool big = wid < a.n_big;
        const int64_t base = big ? (int64_t)wid * a.big_chunks
                                 : (int64_t)a.n_big * a.big_chunks + (int64_t)(wid - a.n_big) * a.arena_chunks;
        A.free_ids = a.free_ids + base;
        A.fc = S->fcache;
        A.base = (int)base; A.cap = big ? a.big_chunks : a.arena_chunks; A.bump = 0; A.g_top = 0; A.fc_n = 0;
    }
    uint4 *stage_w = a.stage + (size_t)wid * 3 * 32 * kWL;          // list L of lane j at + L * 32 * kWL + j * kWL
    uint4 *stage_lane = stage_w + (size_t)lane * kWL;
    uint4 *prec_w = a.prec + (size_t)wid * 32 * kWP;                 // pop t of lane j at + j * kWP + t
    WSide *D = a.side + wid;
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
    const bool dbg = a.dbg != nullptr;
    if (dbg && lane == 0) {
        for (int q = 0; q < kWDbgN; ++q) S->dv[q] = 0;
        S->t_read = clock64();
    }

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
        int wch_b = -1, wch_n = 0;   // bucket whose chunk chain S->wch holds, and its length
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
            const int pend_i = pend ? 1 : 0;
            // early stop (the same for the whole bucket until a hit): the sequential search pops one entry
            if (!c.nonstop && b > best_score + O.s_mm) {
                --n_entries;
                ++pops;
                if (TRACE) {
                    WEnt y = pend ? px : wunpack(chunks[(size_t)S->top_chunk[b] * kWCH + S->top_cnt[b] - 1]);
                    trace = trace_pop<TRACE>(trace, binfo, y, n_entries);
                }
                break;
            }
            if (dbg && lane == 0) S->t_mark = clock64();
            // the wave's entries, in pop order: the pending child (if any), then bucket b from the top
            const int navail = pend_i + S->n_in[b];
            const int Wcap = navail < kWE ? navail : kWE;
            // the bucket's chunks down to the wave's last entry; bucket b gets no pushes while it is popped,
            // so the chain walked for earlier waves of b is still valid below its top
            if (b != wch_b) { wch_b = b; wch_n = 0; }
            int walk_ok = 1, k = wch_n;
            if (lane == 0) {
                const int need = Wcap - pend_i;
                if (k == 0 && need > 0) {
                    if (S->top_chunk[b] < 0) walk_ok = 0;
                    else { S->wch[0] = S->top_chunk[b]; k = 1; }
                }
                int cov = k ? S->top_cnt[b] + (k - 1) * kWCH : 0;
                while (walk_ok && cov < need) {
                    if (k >= kWChain) { walk_ok = 0; break; }
                    const int nx = a.chunk_prev[S->wch[k - 1]];
                    if (nx < 0) { walk_ok = 0; break; }
                    S->wch[k++] = nx;
                    cov += kWCH;
                }
            }
            walk_ok = __shfl_sync(FULL, walk_ok, 0);
            wch_n = __shfl_sync(FULL, k, 0);
            if (!walk_ok) { ret = kErrStack; break; }
            __syncwarp();
            {
                // the bucket's entries come in by asynchronous 16-byte copies, all of a lane's started before it
                // waits once
                const int cnt = S->top_cnt[b];
                for (int e = lane; e < Wcap; e += 32) {
                    if (e < pend_i) S->ent[e] = wpack(px);
                    else {
                        const int d = e - pend_i;
                        int ci, p;
                        if (d < cnt) { ci = 0; p = cnt - 1 - d; }
                        else { const int d2 = d - cnt; ci = 1 + d2 / kWCH; p = kWCH - 1 - d2 % kWCH; }
                        cp_async16(&S->ent[e], chunks + (size_t)S->wch[ci] * kWCH + p);
                    }
                }
                cp_async_wait_all();
            }
            __syncwarp();
            WDBG_LAP(kDbgCycLoad);

            // ---- speculative chains: idle lanes take the next entry, busy lanes pop ----
            int e_next = 0, limit = Wcap;
            int ce = -1;                                   // this lane's entry
            int lp = 0, nl0 = 0, nl1 = 0, nl2 = 0;        // this lane's pops and staged pushes in the wave
            int e_p0 = 0, e_np = 0, e_pre = 0, e_mpre = 0, e_pmax = 0, e_s0 = 0, e_s1 = 0, e_s2 = 0;
            uint32_t e_fs = 0;
            WEnt x;
            x.k = 0; x.l = 0; x.i = 0; x.isdiff = 0; x.n_mm = x.n_gapo = x.n_gape = x.n_ins = 0; x.state = 0;
            WWalk wk;
            wk.k = 0; wk.l = 0; wk.i = 0; wk.f = 0; wk.on = false;
            for (;;) {
                const int nlm = max(nl0, max(nl1, nl2));
                const bool want = ce < 0 && lp + kWGrabPops <= kWP && nlm + 9 * kWGrabPops <= kWL;
                const unsigned wb = __ballot_sync(FULL, want);
                if (wb && e_next < limit) {
                    const int e = e_next + __popc(wb & lt_mask);
                    if (want && e < limit) {
                        ce = e;
                        x = wunpack(S->ent[e]);
                        e_p0 = lp; e_np = 0; e_pre = 0; e_mpre = 0; e_pmax = 0; e_fs = 0;
                        e_s0 = nl0; e_s1 = nl1; e_s2 = nl2;
                    }
                    e_next = min(limit, e_next + __popc(wb));
                }
                if (!__any_sync(FULL, ce >= 0)) break;
                WDBG_ADD(kDbgSteps, 1);
                int stop_e = 0x7fffffff;
                if (ce >= 0) {
                    uint32_t mt = 0;
                    const int endc = lane_step<TRACE, ST>(ix, O, c, S, D, lane, x, wk, b, fetches, stage_lane, tl,
                                                      prec_w + (size_t)lane * kWP, lp, nl0, nl1, nl2, mt);
                    if (endc == -2) goto next_step;          // an exact walk goes on
                    ++e_np;
                    if (e_pre > e_mpre) e_mpre = e_pre;     // n_entries before this pop, relative to the chain start
                    e_pre += (int)(mt & 15u) + (int)((mt >> 4) & 1u) - 1;
                    if (e_pre > e_pmax) e_pmax = e_pre;
                    e_fs += mt >> 5;
                    if (endc >= 0) {
                        S->e_info[ce] = (uint32_t)lane | (uint32_t)e_p0 << 8 | (uint32_t)e_np << 16 | (uint32_t)endc << 24;
                        S->e_seg[0][ce] = (uint16_t)(e_s0 | (nl0 - e_s0) << 8);
                        S->e_seg[1][ce] = (uint16_t)(e_s1 | (nl1 - e_s1) << 8);
                        S->e_seg[2][ce] = (uint16_t)(e_s2 | (nl2 - e_s2) << 8);
                        S->e_a[ce] = ((uint32_t)e_pre & 0xffffu) | (uint32_t)e_mpre << 16;
                        S->e_b[ce] = (uint32_t)e_pmax | e_fs << 16;
                        if (endc > 0) stop_e = ce;
                        ce = -1;
                    }
                }
            next_step:
                // a stop ends the hand-out after its entry; chains past it are dropped
                const int ms = __reduce_min_sync(FULL, stop_e);
                if (ms != 0x7fffffff && ms + 1 < limit) limit = ms + 1;
                if (ce >= limit) { ce = -1; wk.on = false; }
            }
            const int E = min(e_next, limit);
            __syncwarp();
            if (dbg) {
                const unsigned cp = __reduce_add_sync(FULL, (unsigned)lp);
                WDBG_LAP(kDbgCycChain);
                WDBG_ADD(kDbgWaves, 1);
                WDBG_ADD(kDbgLanes, E);
                WDBG_ADD(kDbgChainPops, cp);
            }

            // ---- replay in sequential order. Without the trace hash, the entries before the first one that
            // stops the replay (a hit, an error, an unfinished chain, or the max_entries cut-off inside its
            // chain) are replayed at once from prefix sums; that entry, and in trace mode every entry, one pop
            // at a time. Lane j holds entries kEPL*j .. kEPL*j + kEPL - 1.
            int consumed = 0;
            bool stop = false, search_end = false, new_pend = false;
            int j_first = 0;
            if (!TRACE) {
                int pre_k[kEPL], mpre_k[kEPL], pmax_k[kEPL], np_k[kEPL];
                uint32_t fs_k[kEPL];
                bool hard_k[kEPL];
                int lsum = 0;
#pragma unroll
                for (int k = 0; k < kEPL; ++k) {
                    const int e = kEPL * lane + k;
                    pre_k[k] = mpre_k[k] = pmax_k[k] = np_k[k] = 0; fs_k[k] = 0; hard_k[k] = false;
                    if (e < E) {
                        const uint32_t inf = S->e_info[e], ea = S->e_a[e], eb = S->e_b[e];
                        pre_k[k] = (int)(int16_t)(ea & 0xffffu);
                        mpre_k[k] = (int)(ea >> 16);
                        pmax_k[k] = (int)(eb & 0xffffu);
                        fs_k[k] = eb >> 16;
                        np_k[k] = (int)((inf >> 16) & 0xffu);
                        hard_k[k] = (inf >> 24) != 0;
                    }
                    lsum += pre_k[k];
                }
                int incl = lsum;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += v;
                }
                int run = n_entries + incl - lsum;         // n_entries before this lane's first entry
                int first = 0x7fffffff;
#pragma unroll
                for (int k = 0; k < kEPL; ++k) {
                    const int e = kEPL * lane + k;
                    if (e < E && first == 0x7fffffff && (hard_k[k] || run + mpre_k[k] > O.max_entries)) first = e;
                    run += pre_k[k];
                }
                const int sstar = min(__reduce_min_sync(FULL, first), E);
                run = n_entries + incl - lsum;
                int t_np = 0, t_pre = 0, pk = 0;
                uint32_t t_fs = 0;
#pragma unroll
                for (int k = 0; k < kEPL; ++k) {
                    const int e = kEPL * lane + k;
                    if (e < sstar) {
                        t_np += np_k[k]; t_pre += pre_k[k]; t_fs += fs_k[k];
                        pk = max(pk, run + pmax_k[k]);
                    }
                    run += pre_k[k];
                }
                pops += (uint64_t)__reduce_add_sync(FULL, (unsigned)t_np);
                n_entries += (int)__reduce_add_sync(FULL, (unsigned)t_pre);
                f_alg += __reduce_add_sync(FULL, t_fs);
                const int pkm = (int)__reduce_max_sync(FULL, (unsigned)pk);
                if (pkm > peak) peak = pkm;
                consumed = sstar;
                j_first = sstar;
            }
            for (int e = j_first; e < E && !stop && (TRACE || e == j_first); ++e) {
                const uint32_t inf = S->e_info[e];
                const int ln = (int)(inf & 0xffu), p0 = (int)((inf >> 8) & 0xffu), np = (int)((inf >> 16) & 0xffu);
                const int endc = (int)(inf >> 24);
                // the entry's per-pop data, np <= kWP <= 64 words, one load per lane
                static_assert(kWP <= 64, "replay prefetch");
                const uint32_t m_lo = lane < np ? D->meta[p0 + lane][ln] : 0u;
                const uint32_t m_hi = lane + 32 < np ? D->meta[p0 + lane + 32][ln] : 0u;
                for (int t = 0; t < np; ++t) {
                    if (n_entries > O.max_entries) { search_end = true; stop = true; break; }
                    --n_entries;
                    ++pops;
                    const uint32_t meta = __shfl_sync(FULL, t < 32 ? m_lo : m_hi, t & 31);
                    f_alg += meta >> 5;
                    if (TRACE) trace = trace_pop<TRACE>(trace, binfo, wunpack(prec_w[(size_t)ln * kWP + p0 + t]), n_entries);
                    if (t == np - 1 && endc == 3) { ret = kErrScore; search_end = true; stop = true; break; }
                    if (t == np - 1 && endc == 1) {
                        // the hit, as bwt_match_gap handles it
                        consumed = e + 1;
                        stop = true;
                        WEnt h = wunpack(D->hz[ln]);
                        uint64_t k = D->hk[ln], l = D->hl[ln];
                        int sc = h.n_mm * O.s_mm + h.n_gapo * O.s_gapo + h.n_gape * O.s_gape;
                        int diffs = h.n_mm + h.n_gapo + (c.gape ? h.n_gape : 0);
                        if (n_aln == 0) {
                            best_score = sc;
                            if (!c.nonstop) c.max_diff = diffs + 1 > max_diff0 ? max_diff0 : diffs + 1;
                        }
                        if (sc == best_score) best_cnt = (int)(uint32_t)((uint64_t)(int64_t)best_cnt + (l - k + 1));
                        else if (best_cnt > O.max_top2) { search_end = true; break; }
                        bool add = true;
                        if (h.n_gapo)
                            for (int q = 0; q < n_aln; ++q)
                                if (aln[3 * q + 1] == k && aln[3 * q + 2] == l) { add = false; break; }
                        if (add) {
                            int ldp = h.isdiff ? h.i : 0;
                            uint64_t xx = (uint64_t)(int64_t)(int)(l - k + 1);
                            int jb = 0;
                            for (int t0 = 0; t0 < ldp; t0 += 32) {
                                int tt = t0 + lane;
                                uint64_t v = tt < ldp ? S->W[tt] : 0, wv = v & kW48;
                                bool eq = tt < ldp && wv == xx, gt = tt < ldp && wv > xx;
                                unsigned bal = __ballot_sync(FULL, eq);
                                int rank = __popc(bal & lt_mask);
                                if (gt) S->W[tt] = (v & ~kW48) | (wv - xx);
                                if (eq) S->W[tt] = (1ull << 48) | ((ix.seq_len - (uint64_t)(jb + rank + 1)) & kW48);
                                jb += __popc(bal);
                            }
                            __syncwarp();
                            if (n_aln == a.aln_cap) { ret = kErrAln; search_end = true; break; }
                            if (lane == 0) {
                                int n_del = h.n_gapo + h.n_gape - h.n_ins;
                                aln[3 * n_aln] = (uint64_t)(h.n_mm & 0xff) | (uint64_t)(h.n_gapo & 0xff) << 8
                                               | (uint64_t)(h.n_gape & 0xff) << 16 | (uint64_t)(sc & 0xfffff) << 24
                                               | (uint64_t)(h.n_ins & 0x3ff) << 44 | (uint64_t)(n_del & 0x3ff) << 54;
                                aln[3 * n_aln + 1] = k;
                                aln[3 * n_aln + 2] = l;
                            }
                            __syncwarp();
                            ++n_aln;
                        }
                        break;
                    }
                    n_entries += (int)(meta & 15u) + (int)((meta >> 4) & 1u);
                    if (n_entries > peak) peak = n_entries;
                }
                if (stop) break;
                consumed = e + 1;
                if (endc == 2) { new_pend = true; stop = true; }
            }
            if (dbg) {
                WDBG_LAP(kDbgCycReplay);
                WDBG_ADD(kDbgConsumed, consumed);
                WDBG_ADD(kDbgCont, new_pend ? 1 : 0);
                WDBG_ADD(kDbgHazard, consumed > 0 && (S->e_info[consumed - 1] >> 24) == 1 ? 1 : 0);
            }
            if (search_end) break;
            // take the consumed entries off bucket b (entry 0 may have been the pending child)
            const int C = consumed - pend_i;
            if (C > 0) {
                // whole chunks emptied: wch[0..j); the new top is wch[j], or the chunk below the last walked one
                int cnt = S->top_cnt[b], left = C, j = 0;
                while (j < wch_n && left >= cnt) { left -= cnt; ++j; cnt = kWCH; }
                const int tc = j < wch_n ? S->wch[j] : (j > 0 ? a.chunk_prev[S->wch[j - 1]] : S->top_chunk[b]);
                if (tc < 0 && left > 0) { ret = kErrStack; break; }
                for (int t = 0; t < j; ++t) A.release(S->wch[t], lane);
                // drop them from the kept chain
                const int keep = wch_n - j;
                const int v = lane < keep ? S->wch[j + lane] : 0;
                __syncwarp();
                if (j > 0) {
                    if (keep > 0) { if (lane < keep) S->wch[lane] = v; wch_n = keep; }
                    else { if (lane == 0 && tc >= 0) S->wch[0] = tc; wch_n = tc >= 0 ? 1 : 0; }
                }
                if (lane == 0) {
                    S->top_chunk[b] = tc;
                    S->top_cnt[b] = (uint16_t)(tc >= 0 ? cnt - left : 0);
                    S->n_in[b] -= C;
                    if (S->n_in[b] == 0) S->mask[b >> 5] &= ~(1u << (b & 31));
                }
                __syncwarp();
            }
            pend = false;
            if (new_pend) {
                pend = true;
                pend_b = b;
                px = wunpack(D->lane_x[S->e_info[consumed - 1] & 0xffu]);
            }
            // commit the pushes of the consumed entries, list by list (one list per target bucket), in replay
            // order: entry order, then the order the entry's lane staged them
            bool fail = false;
            for (int L = 0; L < 3 && !fail; ++L) {
                if (lst_pen[L] < 0) continue;
                const int X = b + lst_pen[L];
                int cnt_k[kEPL], lsum = 0;
#pragma unroll
                for (int k = 0; k < kEPL; ++k) {
                    const int e = kEPL * lane + k;
                    cnt_k[k] = e < consumed ? (int)(S->e_seg[L][e] >> 8) : 0;
                    lsum += cnt_k[k];
                }
                int incl = lsum;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(FULL, incl, o);
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
                // inclusive counts per entry (e_a is free after the replay)
                {
                    int run = incl - lsum;
#pragma unroll
                    for (int k = 0; k < kEPL; ++k) {
                        const int e = kEPL * lane + k;
                        run += cnt_k[k];
                        if (e < consumed) S->e_a[e] = (uint32_t)run;
                    }
                }
                __syncwarp();
                // copy: output position p (0..T) comes from the entry e with incl[e-1] <= p < incl[e]. In rounds of
                // kWE positions: each lane starts asynchronous 16-byte copies (cp.async, no registers held) of its
                // positions' staged entries into the wave's entry array (free once the chains are done), waits
                // once for them all, and stores them to the chunks: one memory latency per round instead of one
                // per 32 positions
                const uint4 *stl = stage_w + (size_t)L * 32 * kWL;
                for (int r0 = 0; r0 < T; r0 += kWE) {
                    const int rn = min(T - r0, kWE);
                    int lo = 0;                          // a lane's positions rise, so each search starts at the last
                    for (int t = lane; t < rn; t += 32) {
                        const int p = r0 + t;
                        int hi = consumed - 1;
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if ((int)S->e_a[mid] > p) hi = mid; else lo = mid + 1;
                        }
                        const int before = lo ? (int)S->e_a[lo - 1] : 0;
                        const int ln = (int)(S->e_info[lo] & 0xffu);
                        const int st0 = (int)(S->e_seg[L][lo] & 0xffu);
                        cp_async16(&S->ent[t], stl + (size_t)ln * kWL + st0 + (p - before));
                    }
                    cp_async_wait_all();
                    for (int t = lane; t < rn; t += 32) {   // the same lane's places: no exchange between lanes
                        const int g = cnt0 + r0 + t;
                        const int ci = g / kWCH;
                        const int chunk = c0 >= 0 ? (ci == 0 ? c0 : S->newc[ci - 1]) : S->newc[ci];
                        chunks[(size_t)chunk * kWCH + (g % kWCH)] = S->ent[t];
                    }
                }
                __syncwarp();
                if (lane == 0) {
                    const int last = cnt0 + T - 1;
                    const int ci = last / kWCH;
                    S->top_chunk[X] = c0 >= 0 ? (ci == 0 ? c0 : S->newc[ci - 1]) : S->newc[ci];
                    S->top_cnt[X] = (uint16_t)(last % kWCH + 1);
                    S->n_in[X] += T;
                    S->mask[X >> 5] |= 1u << (X & 31);
                }
                __syncwarp();
            }
            WDBG_LAP(kDbgCycCommit);
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
        S->dv[kDbgReads] = 1;
        S->dv[kDbgPops] = pops;
        const unsigned long long cyc = (unsigned long long)(clock64() - S->t_read);
        S->dv[kDbgCycRead] = cyc;
        for (int q = 0; q < kWDbgN; ++q)
            if (q != kDbgCycReadMax) atomicAdd(a.dbg + q, S->dv[q]);
        atomicMax(a.dbg + kDbgCycReadMax, cyc);
    }
    if (lane == 0) {
        a.out_n[r] = ret;
        a.out_pops[r] = pops;
        a.out_trace[r] = TRACE ? trace : 0;
        a.out_peak[r] = peak;
        a.out_fetch[r] = f_alg;
        a.out_tier[r] = (int8_t)a.tier;
        if (ret == kErrStack && wid >= a.n_big && a.n_big > 0) {
            // to a big warp (its results overwrite these)
            __threadfence();
            const int slot = atomicAdd(a.q_ctl + 1, 1);
            atomicExch(a.ovq + slot, r);
        } else if (ret == kErrStack || ret == kErrAln) a.ovf[atomicAdd(a.ovf_n, 1)] = r;
    }
    __syncwarp();
}

__device__ __forceinline__ uint64_t gtimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// A big warp's next read (lane 0): a queued one first, else one from the list; -1 when the list is done, every
// small warp has finished and the queue is empty, or after a.q_wait_ns of waiting: the reads still queued
// then go to the next pass. If the wait was for a claimed slot whose read id had not arrived, q_ctl[3] is set
// and the host re-runs every read that was ever queued (a read a big warp finished is searched again with the
// same result). A wait of 0 sets q_ctl[3] whenever it gives up, so that path can be exercised on purpose.
__device__ __noinline__ int big_next(const WArgs &a)
{
    volatile int32_t *qc = a.q_ctl;
    const int n_small = a.n_warps - a.n_big;
    const uint64_t t0 = gtimer_ns();
    for (;;) {
        if (gtimer_ns() - t0 > a.q_wait_ns) {
            if (a.q_wait_ns == 0) atomicExch(a.q_ctl + 3, 1);
            return -1;
        }
        const int h = qc[0], t = qc[1];
        if (h < t) {
            if (atomicCAS(a.q_ctl, h, h + 1) == h) {
                // the producer has taken slot h; its read id follows its atomicAdd at once
                for (;;) {
                    const int r = atomicAdd(a.ovq + h, 0);
                    if (r >= 0) { __threadfence(); return r; }
                    if (gtimer_ns() - t0 > a.q_wait_ns) { atomicExch(a.q_ctl + 3, 1); return -1; }
                    __nanosleep(100);
                }
            }
            continue;
        }
        if (*(volatile int32_t *)a.claim < a.n) {
            const int p = atomicAdd(a.claim, 1);
            if (p < a.n) return a.list[p];
            continue;
        }
        if (qc[2] == n_small) {
            __threadfence();
            if (qc[0] >= qc[1]) return -1;
            continue;
        }
        __nanosleep(2000);
    }
}

template <bool TRACE, int ST>
__global__ void __launch_bounds__(32, 16) warp_kernel(const __grid_constant__ WArgs a)
{
    extern __shared__ __align__(16) unsigned char wsm_raw[];
    WarpSmem *S = (WarpSmem *)wsm_raw;
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x;
    if (wid >= a.n_warps) return;
    const bool big = wid < a.n_big;
    for (;;) {
        int r = -1;
        if (lane == 0) {
            if (big) r = big_next(a);
            else {
                const int p = atomicAdd(a.claim, 1);
                r = p < a.n ? a.list[p] : -1;
            }
        }
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r < 0) break;
        warp_read<TRACE, ST>(a, r, wid, S, lane);
    }
    if (!big && a.n_big > 0 && lane == 0) {
        __threadfence();
        atomicAdd(a.q_ctl + 2, 1);
    }
}

}  // namespace galn
