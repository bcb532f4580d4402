// galn_device.cuh -- device side of the `bwa aln` search for sm_100a.
//
// Two occurrence layouts, both one 32-byte sector (one DRAM sector) per block; the kernels take the stride
// as a template parameter and an index holds both.
//   occ64: blocks of 64 symbols of the $-free BWT: four uint32 counts of each base before the block,
//          relative to the block's 2^32-symbol superblock, then the 64 symbols as two 64-bit bit planes
//          (bit j of p0 = low bit of symbol j, of p1 = high bit).
//   occ80: blocks of 80 symbols: three uint32 counts (A, C, G) before the block relative to its superblock
//          of 2^25 blocks, a word holding bits 64-79 of both planes (p0 in the low half, p1 in the high),
//          then bits 0-63 of p0 and p1. The count of T is the position's rank minus the other three.
//          20% smaller (80 MB for a 100 Mbp genome, inside the device's persisting-L2 limit), and a pair
//          (k-1, l) falls in one block more often.
// One LF step for one position is one 32-byte fetch; the reference's layout (src/bwtsearch.h:22-34, 128
// symbols in 64 bytes) needs two sectors. The superblock counts are kernel parameters. Counts and intervals
// are the same integers as bwt_occ / bwt_2occ / bwt_occ4 / bwt_2occ4 (src/bwtsearch.h:46-108,
// src/bwtgap_hd.h:135-192).
#pragma once

#include <stdint.h>

namespace galn {

constexpr int kMaxSuper = 16;          // superblocks: 2^36 symbols for occ64, 2^29 x 80 for occ80
constexpr int kOcc64 = 64, kOcc80 = 80;   // the layouts' strides
constexpr int kOcc80SuperShift = 25;   // occ80 blocks per superblock: 2^25
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

__device__ __forceinline__ uint64_t sel4(int c, uint64_t a0, uint64_t a1, uint64_t a2, uint64_t a3)
{
    uint64_t lo = (c & 1) ? a1 : a0, hi = (c & 1) ? a3 : a2;
    return (c & 2) ? hi : lo;
}

// Occ(c, k1) and Occ(c, l) for all four bases (positions in [-1, seq_len]; Occ(., -1) = 0), without a branch
// around the loads: both blocks are read (the same address twice when k1 and l share a block, which the L1
// merges), so threads of a warp that differ in that respect still wait for one round trip together.
// `fetches` counts the distinct 32-byte blocks (the roofline's unit of algorithmic traffic): one when both
// positions fall in one block.
template <int S>
__device__ __forceinline__ void occ4_pair_u(const IndexView &ix, uint64_t k1, uint64_t l, uint64_t ok[4], uint64_t ol[4],
                                            uint32_t &fetches);

template <>
__device__ __forceinline__ void occ4_pair_u<kOcc64>(const IndexView &ix, uint64_t k1, uint64_t l, uint64_t ok[4],
                                                    uint64_t ol[4], uint32_t &fetches)
{
    const bool kn = k1 == ~0ull, ln = l == ~0ull;
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

// Occ of the four bases up to $-free position p at offset j of occ80 block b (its two uint4 halves c, x)
__device__ __forceinline__ void occ80_counts(const IndexView &ix, uint4 c, uint4 x, uint64_t p, int j, uint64_t b,
                                             uint64_t o[4])
{
    const uint64_t lo0 = (uint64_t)x.x | ((uint64_t)x.y << 32), lo1 = (uint64_t)x.z | ((uint64_t)x.w << 32);
    const uint32_t h0 = c.w & 0xffffu, h1 = c.w >> 16;
    const uint64_t mlo = j >= 63 ? ~0ull : (2ull << j) - 1;
    const uint32_t mhi = j >= 64 ? (2u << (j - 64)) - 1 : 0u;
    const uint64_t *s = ix.sb[b >> kOcc80SuperShift];
    const uint64_t a = s[0] + c.x + __popcll(~lo0 & ~lo1 & mlo) + __popc(~h0 & ~h1 & mhi);
    const uint64_t cc = s[1] + c.y + __popcll(lo0 & ~lo1 & mlo) + __popc(h0 & ~h1 & mhi);
    const uint64_t g = s[2] + c.z + __popcll(~lo0 & lo1 & mlo) + __popc(~h0 & h1 & mhi);
    o[0] = a; o[1] = cc; o[2] = g;
    o[3] = p + 1 - a - cc - g;
}

template <>
__device__ __forceinline__ void occ4_pair_u<kOcc80>(const IndexView &ix, uint64_t k1, uint64_t l, uint64_t ok[4],
                                                    uint64_t ol[4], uint32_t &fetches)
{
    const bool kn = k1 == ~0ull, ln = l == ~0ull;
    const uint64_t pk = kn ? 0 : k1 - (k1 >= ix.primary);
    const uint64_t pl = ln ? 0 : l - (l >= ix.primary);
    const uint64_t bk = pk / 80, bl = pl / 80;
    const bool same = !kn && !ln && bk == bl;
    fetches += same ? 1u : (uint32_t)(!kn) + (uint32_t)(!ln);
    const uint4 *qk = ix.blk + (bk << 1), *ql = ix.blk + (bl << 1);
    const uint4 ck = __ldg(qk), xk = __ldg(qk + 1), cl = __ldg(ql), xl = __ldg(ql + 1);
    occ80_counts(ix, ck, xk, pk, (int)(pk - 80 * bk), bk, ok);
    occ80_counts(ix, cl, xl, pl, (int)(pl - 80 * bl), bl, ol);
    if (kn) { ok[0] = ok[1] = ok[2] = ok[3] = 0; }
    if (ln) { ol[0] = ol[1] = ol[2] = ol[3] = 0; }
}

// (k, l) <- interval of base c prepended: [C(c) + Occ(c, k-1) + 1, C(c) + Occ(c, l)]
template <int S>
__device__ __forceinline__ void extend1(const IndexView &ix, int c, uint64_t &k, uint64_t &l, uint32_t &fetches)
{
    uint64_t ok[4], ol[4];
    occ4_pair_u<S>(ix, k - 1, l, ok, ol, fetches);
    k = ix.C[c] + sel4(c, ok[0], ok[1], ok[2], ok[3]) + 1;
    l = ix.C[c] + sel4(c, ol[0], ol[1], ol[2], ol[3]);
}

__device__ __forceinline__ uint64_t trace_mix(uint64_t h, uint64_t v) { return (h ^ v) * kTracePrime; }

}  // namespace galn
