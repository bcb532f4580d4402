// galn_search.cuh -- one read of bwt_match_gap on one thread (sm_100a).
//
// The algorithm is BWA 0.7.19's bwt_match_gap as the reference runs it (src/bwtgap_hd.h:338-473, and the
// contract of its pop order: lowest score bucket first, last pushed first within a bucket, the
// max_entries test before each pop, early stop at best_score + s_mm unless -N, the -R stop, gapped-hit
// de-duplication by (k, l), gap_shadow on the width array). Results, pop counts and the trace hash are
// the reference's (src/bwtgap_hd.h:80-100).
//
// Device data structures (this implementation's own):
//   * the stack is a set of LIFO lists threaded through a per-thread arena of entries; bucket heads in a
//     per-thread array; a 128-bit register mask of non-empty buckets finds the next bucket after one
//     empties (a scan over the heads above 128 buckets);
//   * an entry is 16 bytes (k and l in 38 bits, i in 16, counts in 7-8 bits; n_del = n_gapo + n_gape -
//     n_ins is not stored; the score is the bucket) unless the batch's options need the 32-byte form;
//   * the light tier allocates entries by bumping a counter (each slot written once, sequentially); the
//     heavy tiers recycle popped slots through a free list so the arena bounds live entries only;
//   * exact-child fusion: with non-negative penalties the exact-match child is the next pop (it has the
//     parent's score, the lowest non-empty bucket, and is pushed last), so it stays in registers instead
//     of going through the arena; n_entries still counts it, so every test sees the same numbers;
//   * width[] and seed_width[] are one uint64 per position (bid << 48 | w).
#pragma once

#include "galn_device.cuh"

namespace galn {

struct Workspace {
    uint4 *ent;             // cap entries of 16 bytes, or cap*2 uint4 for 32-byte entries
    int32_t *link;          // cap
    int32_t *heads;         // hcap per slot
    uint64_t *wid;          // wcap per slot
    uint64_t *aln;          // aln_cap * 3 per slot
    int cap, hcap, wcap, aln_cap;
};

struct SearchResult {
    int ret;
    uint64_t pops, trace;
    int peak;
    uint32_t fetches;
};

constexpr uint64_t kW48 = (1ull << 48) - 1;
constexpr uint64_t kK38 = (1ull << 38) - 1;

__device__ __forceinline__ int next_bucket(uint64_t m0, uint64_t m1, int from)
{
    if (from < 64) {
        uint64_t x = m0 & (~0ull << from);
        if (x) return __ffsll((long long)x) - 1;
        from = 64;
    }
    if (from < 128) {
        uint64_t x = m1 & (~0ull << (from - 64));
        if (x) return 64 + __ffsll((long long)x) - 1;
    }
    return 1 << 30;
}

// bwt_cal_width on the reversed+complemented query (the complement is undone per base)
template <int S = kOcc64>
__device__ __forceinline__ void cal_width(const IndexView &ix, int len, const uint8_t *q, uint64_t *w, uint32_t &fetches)
{
    uint64_t k = 0, l = ix.seq_len;
    uint64_t bid = 0;
    for (int i = 0; i < len; ++i) {
        int c = q[i];
        c = c > 3 ? 4 : 3 - c;
        if (c < 4) extend1<S>(ix, c, k, l, fetches);
        if (k > l || c > 3) { k = 0; l = ix.seq_len; ++bid; }
        w[i] = (bid << 48) | ((l - k + 1) & kW48);
    }
    ++bid;
    w[len] = bid << 48;
}

struct Entry {
    uint64_t k, l;
    uint32_t info;
    int ldp;
    int n_mm, n_gapo, n_gape, state, n_ins, n_del;
};

template <bool WIDE>
__device__ __forceinline__ void store_entry(uint4 *ent, int idx, int score, int i, uint64_t k, uint64_t l, int n_mm,
                                            int n_gapo, int n_gape, int n_ins, int n_del, int state, int is_diff)
{
    if (!WIDE) {
        uint64_t w0 = (k & kK38) | ((uint64_t)(uint32_t)i << 38) | ((uint64_t)(n_mm & 127) << 54)
                    | ((uint64_t)state << 61) | ((uint64_t)(is_diff ? 1 : 0) << 63);
        uint64_t w1 = (l & kK38) | ((uint64_t)(n_gapo & 127) << 38) | ((uint64_t)(n_gape & 127) << 45)
                    | ((uint64_t)(n_ins & 255) << 52);
        ent[idx] = make_uint4((uint32_t)w0, (uint32_t)(w0 >> 32), (uint32_t)w1, (uint32_t)(w1 >> 32));
    } else {
        uint32_t info = (uint32_t)score << 21 | (uint32_t)i;
        uint32_t ldp = is_diff ? (uint32_t)i : 0u;
        uint32_t cnts = (uint32_t)(n_mm & 255) | (uint32_t)(n_gapo & 255) << 8 | (uint32_t)(n_gape & 255) << 16
                      | (uint32_t)(state & 255) << 24;
        uint32_t id = (uint32_t)(n_ins & 0xffff) | (uint32_t)(n_del & 0xffff) << 16;
        ent[2 * idx] = make_uint4((uint32_t)k, (uint32_t)(k >> 32), (uint32_t)l, (uint32_t)(l >> 32));
        ent[2 * idx + 1] = make_uint4(info, ldp, cnts, id);
    }
}

template <bool WIDE>
__device__ __forceinline__ void load_entry(const uint4 *ent, int idx, int score, Entry &e)
{
    if (!WIDE) {
        uint4 v = ent[idx];
        uint64_t w0 = (uint64_t)v.x | ((uint64_t)v.y << 32), w1 = (uint64_t)v.z | ((uint64_t)v.w << 32);
        e.k = w0 & kK38;
        int i = (int)((w0 >> 38) & 0xffff);
        e.n_mm = (int)((w0 >> 54) & 127);
        e.state = (int)((w0 >> 61) & 3);
        e.ldp = (w0 >> 63) ? i : 0;
        e.l = w1 & kK38;
        e.n_gapo = (int)((w1 >> 38) & 127);
        e.n_gape = (int)((w1 >> 45) & 127);
        e.n_ins = (int)((w1 >> 52) & 255);
        e.n_del = e.n_gapo + e.n_gape - e.n_ins;
        e.info = (uint32_t)score << 21 | (uint32_t)i;
    } else {
        uint4 a = ent[2 * idx], b = ent[2 * idx + 1];
        e.k = (uint64_t)a.x | ((uint64_t)a.y << 32);
        e.l = (uint64_t)a.z | ((uint64_t)a.w << 32);
        e.info = b.x;
        e.ldp = (int)b.y;
        e.n_mm = (int)(b.z & 255); e.n_gapo = (int)((b.z >> 8) & 255); e.n_gape = (int)((b.z >> 16) & 255);
        e.state = (int)(b.z >> 24);
        e.n_ins = (int)(b.w & 0xffff); e.n_del = (int)(b.w >> 16);
    }
}

// One read. q: reversed+complemented codes (0..3, 4 ambiguous). W / SW: width and seed width, already
// computed. Records go to aln (3 uint64 each). Returns the search result (n_aln or an error code).
template <bool WIDE, bool FREELIST, bool TRACE, int S = kOcc64>
__device__ SearchResult match_gap(const IndexView &ix, const BatchOpt &O, int max_diff0, int len, const uint8_t *q,
                                  uint64_t *W, uint64_t *SW, bool use_seed, const Workspace &ws, int slot,
                                  uint32_t fetches)
{
    SearchResult R;
    R.pops = 0; R.trace = kTraceInit; R.peak = 0; R.ret = 0; R.fetches = fetches;
    uint4 *ent = ws.ent + (size_t)slot * ws.cap * (WIDE ? 2 : 1);
    int32_t *link = ws.link + (size_t)slot * ws.cap;
    int32_t *heads = ws.heads + (size_t)slot * ws.hcap;
    uint64_t *aln = ws.aln + (size_t)slot * ws.aln_cap * 3;
    const int n_stacks = O.n_stacks;
    const int s_mm = O.s_mm, s_gapo = O.s_gapo, s_gape = O.s_gape;
    const bool gape = (O.mode & kModeGape) != 0;
    const bool nonstop = (O.mode & kModeNonstop) != 0;
    const bool fuse = s_mm >= 0 && s_gapo >= 0 && s_gape >= 0;
    const bool small_mask = n_stacks <= 128;
    const int seed_len = len > O.seed_len ? O.seed_len : 0x7fffffff;   // as the read's local option

    int best_score = (max_diff0 + 1) * s_mm + (O.max_gapo + 1) * s_gapo + (O.max_gape + 1) * s_gape;
    int max_diff = max_diff0, best_cnt = 0, n_aln = 0;

    int n_amb = 0;
    for (int j = 0; j < len; ++j) n_amb += q[j] > 3;
    if (n_amb > max_diff) return R;

    for (int b = 0; b < n_stacks; ++b) heads[b] = -1;
    uint64_t m0 = 0, m1 = 0;
    int best = n_stacks, n_entries = 0, top = 0, free_head = -1, peak = 0;
    uint64_t pops = 0, trace = kTraceInit;

#define GALN_PUSH(SCORE, I, K, L, NMM, NGO, NGE, NIN, NDE, ST, DIFF)                                   \
    do {                                                                                             \
        int sc_ = (SCORE);                                                                           \
        if ((unsigned)sc_ >= (unsigned)n_stacks) { R.ret = kErrScore; goto done; }                   \
        int idx_;                                                                                    \
        if (FREELIST && free_head >= 0) { idx_ = free_head; free_head = link[idx_]; }                \
        else if (top < ws.cap) idx_ = top++;                                                          \
        else { R.ret = kErrStack; goto done; }                                                       \
        store_entry<WIDE>(ent, idx_, sc_, (I), (K), (L), (NMM), (NGO), (NGE), (NIN), (NDE), (ST), (DIFF)); \
        link[idx_] = heads[sc_];                                                                     \
        heads[sc_] = idx_;                                                                           \
        if (sc_ < 64) m0 |= 1ull << sc_; else if (sc_ < 128) m1 |= 1ull << (sc_ - 64);               \
        if (++n_entries > peak) peak = n_entries;                                                    \
        if (sc_ < best) best = sc_;                                                                  \
    } while (0)

    {
        GALN_PUSH(0, len, 0, ix.seq_len, 0, 0, 0, 0, 0, kStM, 0);
        bool pend = false;
        Entry e;
        int e_score = 0;
        // The exact walk of a pop with no difference left (bwt_match_exact_alt) goes one LF step per loop
        // iteration and shares the iteration's one fetch, so that threads of a warp in a walk and threads
        // expanding a pop wait for memory together.
        bool walking = false;
        uint64_t wk = 0, wl = 0;
        int wi = 0;
        int diffs = 0, m = 0, m_seed = 0;
        uint64_t hk = 0, hl = 0;        // the interval of a hit
        for (;;) {
            uint64_t k1, l1;            // this iteration's Occ positions
            int i = 0;
            if (!walking) {
                if (!n_entries) break;
                if (n_entries > O.max_entries) break;
                if (pend) {
                    pend = false;
                    --n_entries;
                } else {
                    int b = best;
                    int idx = heads[b];
                    load_entry<WIDE>(ent, idx, b, e);
                    e_score = b;
                    int nx = link[idx];
                    heads[b] = nx;
                    if (FREELIST) { link[idx] = free_head; free_head = idx; }
                    --n_entries;
                    if (nx < 0) {
                        if (b < 64) m0 &= ~(1ull << b); else if (b < 128) m1 &= ~(1ull << (b - 64));
                        if (n_entries) {
                            if (small_mask) best = next_bucket(m0, m1, b + 1);
                            else { int t = b + 1; while (t < n_stacks && heads[t] < 0) ++t; best = t; }
                        } else best = n_stacks;
                    }
                }
                ++pops;
                if (TRACE) {
                    uint64_t h = trace;
                    h = trace_mix(h, e.info);
                    h = trace_mix(h, e.k);
                    h = trace_mix(h, e.l);
                    h = trace_mix(h, (uint64_t)((uint32_t)(e.n_mm & 255) | (uint32_t)(e.n_gapo & 255) << 8
                                                | (uint32_t)(e.n_gape & 255) << 16 | (uint32_t)(e.state & 255) << 24));
                    h = trace_mix(h, (uint64_t)(e.n_ins & 0xffff) | (uint64_t)(e.n_del & 0xffff) << 16);
                    h = trace_mix(h, (uint64_t)(uint32_t)e.ldp);
                    h = trace_mix(h, (uint64_t)(uint32_t)n_entries);
                    trace = h;
                }
                i = (int)(e.info & 0xffff);
                if (!nonstop && (e.info >> 21) > (uint32_t)(best_score + s_mm)) break;
                diffs = e.n_mm + e.n_gapo + (gape ? e.n_gape : 0);
                m = max_diff - diffs;
                if (m < 0) continue;
                m_seed = use_seed ? O.max_seed_diff - diffs : 0;
                if (i > 0 && m < (int)(W[i - 1] >> 48)) continue;
                if (i == 0) { hk = e.k; hl = e.l; goto hit; }
                if (m == 0 && (e.state == kStM || gape || e.n_gape == O.max_gape)) {
                    // bwt_match_exact_alt over positions i-1 .. 0
                    if (q[i - 1] > 3) continue;
                    walking = true; wk = e.k; wl = e.l; wi = i;
                    k1 = wk - 1; l1 = wl;
                } else {
                    k1 = e.k - 1; l1 = e.l;
                }
            } else {
                if (q[wi - 1] > 3) { walking = false; continue; }
                k1 = wk - 1; l1 = wl;
            }
            {
                uint64_t ck[4], cl[4];
                occ4_pair_u<S>(ix, k1, l1, ck, cl, fetches);
                if (walking) {
                    const int c = q[wi - 1];
                    const uint64_t kk = ix.C[c] + sel4(c, ck[0], ck[1], ck[2], ck[3]) + 1;
                    const uint64_t ll = ix.C[c] + sel4(c, cl[0], cl[1], cl[2], cl[3]);
                    if (kk > ll) { walking = false; continue; }
                    wk = kk; wl = ll;
                    if (--wi > 0) continue;
                    walking = false;
                    hk = wk; hl = wl;
                    goto hit;
                }
                const uint64_t k = e.k, l = e.l;
                --i;
                // child intervals of the four bases, in registers
                const uint64_t kk0 = ix.C[0] + ck[0] + 1, ll0 = ix.C[0] + cl[0];
                const uint64_t kk1 = ix.C[1] + ck[1] + 1, ll1 = ix.C[1] + cl[1];
                const uint64_t kk2 = ix.C[2] + ck[2] + 1, ll2 = ix.C[2] + cl[2];
                const uint64_t kk3 = ix.C[3] + ck[3] + 1, ll3 = ix.C[3] + cl[3];
                uint64_t occ = l - k + 1;
                int allow_diff = 1, allow_M = 1;
                if (i > 0) {
                    uint64_t wa = W[i - 1], wb = W[i];
                    int ba = (int)(wa >> 48), bb = (int)(wb >> 48);
                    if (ba > m - 1) allow_diff = 0;
                    else if (ba == m - 1 && bb == m - 1 && (wa & kW48) == (wb & kW48)) allow_M = 0;
                    int ii = i - (len - seed_len);
                    if (use_seed && ii > 0) {
                        uint64_t sa = SW[ii - 1], sb = SW[ii];
                        int sba = (int)(sa >> 48), sbb = (int)(sb >> 48);
                        if (sba > m_seed - 1) allow_diff = 0;
                        else if (sba == m_seed - 1 && sbb == m_seed - 1 && (sa & kW48) == (sb & kW48)) allow_M = 0;
                    }
                }
                int gaps = e.n_gapo + e.n_gape;
                int tmp = (O.mode & kModeLoggap) ? (gaps ? (31 - __clz(gaps)) : 0) / 2 + 1 : gaps;
                const int b0 = e_score;
                if (!WIDE && !FREELIST && fuse) {
                    // All pushes of this pop at once, in bwt_match_gap's order (src/bwtgap_hd.h:426-470): the
                    // gap children (the kept-interval insertion, then deletions by base) to bucket gb, then the
                    // mismatches (child base (base + j) & 3, j = 1..4) to bucket mb. Entries are taken from the
                    // bump pointer, so a push's place and its bucket link follow from its rank: no per-push branch
                    // and no chain of head loads. The checks come in the order the sequential pushes meet them.
                    const bool indel = allow_diff && i >= O.indel_end_skip + tmp && len - i >= O.indel_end_skip + tmp;
                    const bool st_m = e.state == kStM;
                    const bool open_ok = indel && st_m && e.n_gapo < O.max_gapo;
                    const bool ext_i = indel && e.state == kStI && e.n_gape < O.max_gape;
                    const bool ext_d = indel && e.state == kStD && e.n_gape < O.max_gape
                                       && (gaps < max_diff || occ < (uint64_t)(int64_t)O.max_del_occ);
                    const uint32_t ex = (kk0 <= ll0 ? 1u : 0u) | (kk1 <= ll1 ? 2u : 0u) | (kk2 <= ll2 ? 4u : 0u)
                                      | (kk3 <= ll3 ? 8u : 0u);
                    const uint32_t gs = ((open_ok || ext_i) ? 1u : 0u) | ((open_ok || ext_d) ? ex << 1 : 0u);
                    const int base = q[i];
                    // mismatch j has bit j-1 of msm; child base c has bit (c - base - 1) & 3 (j = 4, the read's own
                    // base, is a mismatch only where that base is ambiguous)
                    uint32_t msm = ((ex | (ex << 4)) >> ((base + 1) & 3)) & 0xfu;
                    if (base <= 3) msm &= 0x7u;
                    if (!(allow_diff && allow_M)) msm = 0;
                    const int ng = __popc(gs), nm = __popc(msm);
                    const int gb = b0 + (st_m ? s_gapo : s_gape), mb = b0 + s_mm;
                    if (ng && (unsigned)gb >= (unsigned)n_stacks) { R.ret = kErrScore; goto done; }
                    if (top + ng > ws.cap) { R.ret = kErrStack; goto done; }
                    if (nm && (unsigned)mb >= (unsigned)n_stacks) { R.ret = kErrScore; goto done; }
                    if (top + ng + nm > ws.cap) { R.ret = kErrStack; goto done; }
                    if (ng) {
                        const int h = heads[gb];
                        const int go = st_m ? 1 : 0, ge = st_m ? 0 : 1;
#pragma unroll
                        for (int t = 0; t < 5; ++t) {
                            if (!(gs & (1u << t))) continue;
                            const int r = __popc(gs & ((1u << t) - 1u));
                            const int idx = top + r;
                            if (t == 0)
                                store_entry<false>(ent, idx, gb, i, k, l, e.n_mm, e.n_gapo + go, e.n_gape + ge,
                                                   e.n_ins + 1, e.n_del, kStI, 1);
                            else
                                store_entry<false>(ent, idx, gb, i + 1, sel4(t - 1, kk0, kk1, kk2, kk3),
                                                   sel4(t - 1, ll0, ll1, ll2, ll3), e.n_mm, e.n_gapo + go,
                                                   e.n_gape + ge, e.n_ins, e.n_del + 1, kStD, 1);
                            link[idx] = r ? idx - 1 : h;
                        }
                        heads[gb] = top + ng - 1;
                        if (gb < 64) m0 |= 1ull << gb; else if (gb < 128) m1 |= 1ull << (gb - 64);
                        if (gb < best) best = gb;
                        top += ng;
                    }
                    if (nm) {
                        const int h = heads[mb];
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            const int bq = (c - base - 1) & 3;
                            if (!(msm & (1u << bq))) continue;
                            const int r = __popc(msm & ((1u << bq) - 1u));
                            const int idx = top + r;
                            store_entry<false>(ent, idx, mb, i, sel4(c, kk0, kk1, kk2, kk3), sel4(c, ll0, ll1, ll2, ll3),
                                               e.n_mm + 1, e.n_gapo, e.n_gape, e.n_ins, e.n_del, kStM, 1);
                            link[idx] = r ? idx - 1 : h;
                        }
                        heads[mb] = top + nm - 1;
                        if (mb < 64) m0 |= 1ull << mb; else if (mb < 128) m1 |= 1ull << (mb - 64);
                        if (mb < best) best = mb;
                        top += nm;
                    }
                    n_entries += ng + nm;
                    // the exact child is the next pop
                    if (base < 4 && ((ex >> base) & 1u)) {
                        e.k = sel4(base, kk0, kk1, kk2, kk3); e.l = sel4(base, ll0, ll1, ll2, ll3);
                        e.info = (uint32_t)b0 << 21 | (uint32_t)i; e.ldp = 0; e.state = kStM;
                        ++n_entries;
                        pend = true;
                    }
                    if (n_entries > peak) peak = n_entries;
                    continue;
                }
                if (allow_diff && i >= O.indel_end_skip + tmp && len - i >= O.indel_end_skip + tmp) {
                    if (e.state == kStM) {
                        if (e.n_gapo < O.max_gapo) {
                            GALN_PUSH(b0 + s_gapo, i, k, l, e.n_mm, e.n_gapo + 1, e.n_gape, e.n_ins + 1, e.n_del, kStI, 1);
#pragma unroll
                            for (int c = 0; c < 4; ++c) {
                                uint64_t kk = sel4(c, kk0, kk1, kk2, kk3), ll = sel4(c, ll0, ll1, ll2, ll3);
                                if (kk <= ll)
                                    GALN_PUSH(b0 + s_gapo, i + 1, kk, ll, e.n_mm, e.n_gapo + 1, e.n_gape, e.n_ins, e.n_del + 1, kStD, 1);
                            }
                        }
                    } else if (e.state == kStI) {
                        if (e.n_gape < O.max_gape)
                            GALN_PUSH(b0 + s_gape, i, k, l, e.n_mm, e.n_gapo, e.n_gape + 1, e.n_ins + 1, e.n_del, kStI, 1);
                    } else if (e.state == kStD) {
                        if (e.n_gape < O.max_gape && (gaps < max_diff || occ < (uint64_t)(int64_t)O.max_del_occ)) {
#pragma unroll
                            for (int c = 0; c < 4; ++c) {
                                uint64_t kk = sel4(c, kk0, kk1, kk2, kk3), ll = sel4(c, ll0, ll1, ll2, ll3);
                                if (kk <= ll)
                                    GALN_PUSH(b0 + s_gape, i + 1, kk, ll, e.n_mm, e.n_gapo, e.n_gape + 1, e.n_ins, e.n_del + 1, kStD, 1);
                            }
                        }
                    }
                }
                const int base = q[i];
                if (allow_diff && allow_M) {
#pragma unroll
                    for (int j = 1; j <= 4; ++j) {
                        int c = (base + j) & 3;
                        int mm = j != 4 || base > 3;
                        uint64_t kk = sel4(c, kk0, kk1, kk2, kk3), ll = sel4(c, ll0, ll1, ll2, ll3);
                        if (kk <= ll) {
                            if (!mm && fuse) {
                                e.k = kk; e.l = ll; e.info = (uint32_t)b0 << 21 | (uint32_t)i; e.ldp = 0; e.state = kStM;
                                ++n_entries; if (n_entries > peak) peak = n_entries;
                                pend = true;
                            } else
                                GALN_PUSH(b0 + (mm ? s_mm : 0), i, kk, ll, e.n_mm + mm, e.n_gapo, e.n_gape, e.n_ins, e.n_del, kStM, mm);
                        }
                    }
                } else if (base < 4) {
                    uint64_t kk = sel4(base, kk0, kk1, kk2, kk3), ll = sel4(base, ll0, ll1, ll2, ll3);
                    if (kk <= ll) {
                        if (fuse) {
                            e.k = kk; e.l = ll; e.info = (uint32_t)b0 << 21 | (uint32_t)i; e.ldp = 0; e.state = kStM;
                            ++n_entries; if (n_entries > peak) peak = n_entries;
                            pend = true;
                        } else
                            GALN_PUSH(b0, i, kk, ll, e.n_mm, e.n_gapo, e.n_gape, e.n_ins, e.n_del, kStM, 0);
                    }
                }
                continue;
            }
        hit:
            {
                const uint64_t k = hk, l = hl;
                int sc = e.n_mm * s_mm + e.n_gapo * s_gapo + e.n_gape * s_gape;
                if (n_aln == 0) {
                    best_score = sc;
                    if (!nonstop) max_diff = diffs + 1 > max_diff0 ? max_diff0 : diffs + 1;
                }
                if (sc == best_score) best_cnt = (int)(uint32_t)((uint64_t)(int64_t)best_cnt + (l - k + 1));
                else if (best_cnt > O.max_top2) break;
                bool add = true;
                if (e.n_gapo) {
                    for (int j = 0; j < n_aln; ++j)
                        if (aln[3 * j + 1] == k && aln[3 * j + 2] == l) { add = false; break; }
                }
                if (add) {
                    // gap_shadow(l - k + 1, ...) with its int argument
                    int x = (int)(l - k + 1);
                    uint64_t xx = (uint64_t)(int64_t)x;
                    int jj = 0;
                    for (int t = 0; t < e.ldp; ++t) {
                        uint64_t v = W[t], wv = v & kW48;
                        if (wv > xx) W[t] = (v & ~kW48) | (wv - xx);
                        else if (wv == xx) { W[t] = (1ull << 48) | ((ix.seq_len - (uint64_t)(++jj)) & kW48); }
                    }
                    if (n_aln == ws.aln_cap) { R.ret = kErrAln; goto done; }
                    aln[3 * n_aln] = (uint64_t)(e.n_mm & 0xff) | (uint64_t)(e.n_gapo & 0xff) << 8
                                   | (uint64_t)(e.n_gape & 0xff) << 16 | (uint64_t)(sc & 0xfffff) << 24
                                   | (uint64_t)(e.n_ins & 0x3ff) << 44 | (uint64_t)(e.n_del & 0x3ff) << 54;
                    aln[3 * n_aln + 1] = k;
                    aln[3 * n_aln + 2] = l;
                    ++n_aln;
                }
            }
        }
        R.ret = n_aln;
    }
done:
#undef GALN_PUSH
    R.pops = pops; R.trace = trace; R.peak = peak; R.fetches = fetches;
    return R;
}

}  // namespace galn
