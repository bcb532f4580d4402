// galn_device.cuh -- device side of the `bwa aln` search for sm_100a.
//
// Occurrence layout ("occ64"): the $-free BWT is cut into blocks of 64 symbols; block b is 32 bytes
// (one DRAM sector): four uint32 counts of each base before the block, relative to the block's
// 2^32-symbol superblock, then the 64 symbols as two 64-bit bit planes (bit j of p0 = low bit of symbol j,
// of p1 = high bit). One LF step for one position is one 32-byte fetch and at most four popcounts; the
// reference's layout (src/bwtsearch.h:22-34, 128 symbols in 64 bytes) needs two sectors. The superblock
// counts (Occ before each 2^32 symbols) are kernel parameters. Counts and intervals are the same integers
// as bwt_occ / bwt_2occ / bwt_occ4 / bwt_2occ4 (src/bwtsearch.h:46-108, src/bwtgap_hd.h:135-192).
#pragma once

#include <stdint.h>

namespace galn {

constexpr int kMaxSuper = 16;          // 2^36 symbols
constexpr int kModeGape = 0x01, kModeLoggap = 0x04, kModeNonstop = 0x10;
constexpr int kStM = 0, kStI = 1, kStD = 2;
constexpr int kErrStack = -1, kErrAln = -2, kErrScore = -3;
constexpr uint64_t kTraceInit = 1469598103934665603ULL;
constexpr uint64_t kTracePrime = 1099511628211ULL;

struct IndexView {
    const uint4 *blk;                   // 2 x uint4 per block
    uint64_t primary, seq_len;
    uint64_t C[4];                      // L2[0..3]
    uint64_t sb[kMaxSuper][4];          // Occ before each superblock
};

// per-batch options as the search uses them (the batch's local gap_opt_t, src/aln_host.c:23-38)
struct BatchOpt {
    int s_mm, s_gapo, s_gape, mode;
    int indel_end_skip, max_del_occ, max_entries;
    int max_diff, max_gapo, max_gape, max_seed_diff, seed_len, max_top2;
    int n_stacks;
    int wide;                           // 1: counts or lengths too large for the 16-byte entry
    int pad_;
};

__device__ __forceinline__ void load_block(const IndexView &ix, uint64_t p, uint4 &cnt, uint64_t &p0, uint64_t &p1)
{
    const uint4 *b = ix.blk + ((p >> 6) << 1);
    cnt = __ldg(b);
    uint4 bits = __ldg(b + 1);
    p0 = (uint64_t)bits.x | ((uint64_t)bits.y << 32);
    p1 = (uint64_t)bits.z | ((uint64_t)bits.w << 32);
}

__device__ __forceinline__ uint64_t base_mask(uint64_t p0, uint64_t p1, int c)
{
    uint64_t a = (c & 1) ? p0 : ~p0;
    uint64_t b = (c & 2) ? p1 : ~p1;
    return a & b;
}

__device__ __forceinline__ uint32_t cnt_of(const uint4 &v, int c)
{
    return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}

// Occ(c, pos) for all four bases; pos in [-1, seq_len]
__device__ __forceinline__ void occ4_one(const IndexView &ix, uint64_t pos, uint64_t o[4])
{
    if (pos == ~0ull) { o[0] = o[1] = o[2] = o[3] = 0; return; }
    uint64_t p = pos - (pos >= ix.primary);
    uint4 cnt; uint64_t p0, p1;
    load_block(ix, p, cnt, p0, p1);
    uint64_t m = (2ull << (p & 63)) - 1;
    const uint64_t *s = ix.sb[p >> 32];
    o[0] = s[0] + cnt.x + __popcll(~p0 & ~p1 & m);
    o[1] = s[1] + cnt.y + __popcll(p0 & ~p1 & m);
    o[2] = s[2] + cnt.z + __popcll(~p0 & p1 & m);
    o[3] = s[3] + cnt.w + __popcll(p0 & p1 & m);
}

// Occ(c, k1) and Occ(c, l) for all four bases, without a branch around the loads: both blocks are read (the
// same address twice when k1 and l share a block, which the L1 merges), so threads of a warp that differ in
// that respect still wait for one round trip together. `fetches` counts the distinct 32-byte blocks (the
// roofline's unit of algorithmic traffic): one when both positions fall in one block.
__device__ __forceinline__ void occ4_pair_u(const IndexView &ix, uint64_t k1, uint64_t l, uint64_t ok[4], uint64_t ol[4],
                                            uint32_t &fetches)
{
    const bool kn = k1 == ~0ull, ln = l == ~0ull;   // Occ(., -1) = 0
    const uint64_t pk = kn ? 0 : k1 - (k1 >= ix.primary);
    const uint64_t pl = ln ? 0 : l - (l >= ix.primary);
    const bool same = !kn && !ln && (pk >> 6) == (pl >> 6);
    fetches += same ? 1u : (uint32_t)(!kn) + (uint32_t)(!ln);
    const uint4 *bk = ix.blk + ((pk >> 6) << 1), *bl = ix.blk + ((pl >> 6) << 1);
    const uint4 ck = __ldg(bk), xk = __ldg(bk + 1), cl = __ldg(bl), xl = __ldg(bl + 1);
    const uint64_t p0k = (uint64_t)xk.x | ((uint64_t)xk.y << 32), p1k = (uint64_t)xk.z | ((uint64_t)xk.w << 32);
    const uint64_t p0l = (uint64_t)xl.x | ((uint64_t)xl.y << 32), p1l = (uint64_t)xl.z | ((uint64_t)xl.w << 32);
    const uint64_t mk = kn ? 0 : (2ull << (pk & 63)) - 1, ml = ln ? 0 : (2ull << (pl & 63)) - 1;
    const uint64_t *sk = ix.sb[pk >> 32], *sl = ix.sb[pl >> 32];
    ok[0] = kn ? 0 : sk[0] + ck.x + __popcll(~p0k & ~p1k & mk);
    ok[1] = kn ? 0 : sk[1] + ck.y + __popcll(p0k & ~p1k & mk);
    ok[2] = kn ? 0 : sk[2] + ck.z + __popcll(~p0k & p1k & mk);
    ok[3] = kn ? 0 : sk[3] + ck.w + __popcll(p0k & p1k & mk);
    ol[0] = ln ? 0 : sl[0] + cl.x + __popcll(~p0l & ~p1l & ml);
    ol[1] = ln ? 0 : sl[1] + cl.y + __popcll(p0l & ~p1l & ml);
    ol[2] = ln ? 0 : sl[2] + cl.z + __popcll(~p0l & p1l & ml);
    ol[3] = ln ? 0 : sl[3] + cl.w + __popcll(p0l & p1l & ml);
}

// Occ(c, k1) and Occ(c, l) for all four bases, one fetch when both fall in one block. `fetches` counts the
// 32-byte blocks read (the roofline's unit of algorithmic traffic).
__device__ __forceinline__ void occ4_pair(const IndexView &ix, uint64_t k1, uint64_t l, uint64_t ok[4], uint64_t ol[4],
                                          uint32_t &fetches)
{
    if (k1 != ~0ull) {
        uint64_t pk = k1 - (k1 >= ix.primary), pl = l - (l >= ix.primary);
        if ((pk >> 6) == (pl >> 6)) {
            ++fetches;
            uint4 cnt; uint64_t p0, p1;
            load_block(ix, pk, cnt, p0, p1);
            uint64_t mk = (2ull << (pk & 63)) - 1, ml = (2ull << (pl & 63)) - 1;
            const uint64_t *s = ix.sb[pk >> 32];
            uint64_t a = ~p0 & ~p1, c = p0 & ~p1, g = ~p0 & p1, t = p0 & p1;
            ok[0] = s[0] + cnt.x + __popcll(a & mk); ol[0] = s[0] + cnt.x + __popcll(a & ml);
            ok[1] = s[1] + cnt.y + __popcll(c & mk); ol[1] = s[1] + cnt.y + __popcll(c & ml);
            ok[2] = s[2] + cnt.z + __popcll(g & mk); ol[2] = s[2] + cnt.z + __popcll(g & ml);
            ok[3] = s[3] + cnt.w + __popcll(t & mk); ol[3] = s[3] + cnt.w + __popcll(t & ml);
            return;
        }
    }
    fetches += (k1 != ~0ull) + (l != ~0ull);
    occ4_one(ix, k1, ok);
    occ4_one(ix, l, ol);
}

// Occ(c, pos) for one base
__device__ __forceinline__ uint64_t occ1(const IndexView &ix, uint64_t pos, int c)
{
    if (pos == ~0ull) return 0;
    uint64_t p = pos - (pos >= ix.primary);
    uint4 cnt; uint64_t p0, p1;
    load_block(ix, p, cnt, p0, p1);
    uint64_t m = (2ull << (p & 63)) - 1;
    return ix.sb[p >> 32][c] + cnt_of(cnt, c) + __popcll(base_mask(p0, p1, c) & m);
}

// (k, l) <- interval of base c prepended: [C(c) + Occ(c, k-1) + 1, C(c) + Occ(c, l)]
__device__ __forceinline__ void extend1(const IndexView &ix, int c, uint64_t &k, uint64_t &l, uint32_t &fetches)
{
    uint64_t k1 = k - 1;
    uint64_t ok, ol;
    if (k1 != ~0ull) {
        uint64_t pk = k1 - (k1 >= ix.primary), pl = l - (l >= ix.primary);
        if ((pk >> 6) == (pl >> 6)) {
            ++fetches;
            uint4 cnt; uint64_t p0, p1;
            load_block(ix, pk, cnt, p0, p1);
            uint64_t bm = base_mask(p0, p1, c);
            uint64_t base = ix.sb[pk >> 32][c] + cnt_of(cnt, c);
            ok = base + __popcll(bm & ((2ull << (pk & 63)) - 1));
            ol = base + __popcll(bm & ((2ull << (pl & 63)) - 1));
            k = ix.C[c] + ok + 1;
            l = ix.C[c] + ol;
            return;
        }
    }
    fetches += (k1 != ~0ull) + (l != ~0ull);
    ok = occ1(ix, k1, c);
    ol = occ1(ix, l, c);
    k = ix.C[c] + ok + 1;
    l = ix.C[c] + ol;
}

__device__ __forceinline__ uint64_t trace_mix(uint64_t h, uint64_t v) { return (h ^ v) * kTracePrime; }

}  // namespace galn
