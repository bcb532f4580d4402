// galn_build_index.cu -- `galn index` on the GPU: the .bwt and .sa files of bwa index 0.7.19 for the text
// T = F . revcomp(F) of a forward sequence F (codes 0..3).
//
// The reference builds them in src/index/gpu_index.cu:1-20 (BWT of T$ by libcubwt or its rank-based sorter,
// then pack + interleaved Occ on the GPU, SA samples by LF walks and list ranking). This builder:
//   1. sorts the suffixes by prefix doubling, refining only the groups still unsorted (Larsson-Sadakane):
//      the first round sorts 21-symbol prefixes (3 bits a symbol, 0 past the end); round r sorts the
//      unsorted suffixes i by (rank of i, rank of i + h), h = 21 * 2^(r-1), where a rank is the suffix-array
//      index of the first suffix of its group. Every sort is a stable LSD radix sort written here: 8-bit
//      digits, per-tile histogram, scan, and a scatter that ranks each tile's items in shared memory so
//      each digit's run leaves the tile as one contiguous write;
//   2. takes the BWT from the suffix array kept on the device, packs it 2 bits a symbol with the Occ counts
//      every 128 symbols (the .bwt layout of bwt_bwtupdate_core, src/index/idxcommon.c:72-112);
//   3. gathers every 32nd suffix-array row (the .sa layout, src/index/idxcommon.c:137-153).
// Positions are 32-bit: texts up to 2^32 - 64 symbols (references up to about 2.1 Gbp), about 38 bytes of
// device memory per symbol at the peak. Everything but the file writes runs on the device.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "galn_internal.h"

namespace galn {
namespace ixb {

constexpr int kRThreads = 512, kRItems = 8, kRTile = kRThreads * kRItems, kRWarps = kRThreads / 32;
constexpr int kScanThreads = 256;
constexpr int kPrefix = 21;            // symbols in a first-round key
constexpr int kMaxRounds = 40;         // h = 21 * 2^39 exceeds any 32-bit text

struct U4 {
    uint64_t c[4];
};
__host__ __device__ inline U4 operator+(const U4 &a, const U4 &b)
{
    return U4{{a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2], a.c[3] + b.c[3]}};
}

// items a scan thread holds: 8 of 4- or 8-byte types, 2 of the 32-byte per-block counts
template <class T>
constexpr int scan_items() { return sizeof(T) > 8 ? 2 : 8; }
template <class T>
constexpr int scan_tile_n() { return kScanThreads * scan_items<T>(); }

template <class T>
struct OpSum {
    __device__ static T id() { return T{}; }
    __device__ static T op(const T &a, const T &b) { return a + b; }
};
template <class T>
struct OpMax {
    __device__ static T id() { return T(0); }
    __device__ static T op(const T &a, const T &b) { return a > b ? a : b; }
};

// ---- scans (reduce, scan of the tile sums, scan of each tile with its carry-in) ----

template <class T, class Op>
__global__ void __launch_bounds__(kScanThreads) scan_reduce(const T *__restrict__ x, uint64_t n, T *__restrict__ part)
{
    constexpr int kItems = scan_items<T>(), kTile = scan_tile_n<T>();
    __shared__ T s[kScanThreads];
    const int t = threadIdx.x;
    const uint64_t base = (uint64_t)blockIdx.x * kTile;
    T acc = Op::id();
    for (int j = 0; j < kItems; ++j) {
        const uint64_t i = base + (uint64_t)j * kScanThreads + t;
        if (i < n) acc = Op::op(acc, x[i]);
    }
    s[t] = acc;
    __syncthreads();
    for (int w = kScanThreads / 2; w > 0; w >>= 1) {
        if (t < w) s[t] = Op::op(s[t], s[t + w]);
        __syncthreads();
    }
    if (t == 0) part[blockIdx.x] = s[0];
}

// In place: inclusive (INCL) or exclusive scan of one tile, offset by carry[tile] when carry is given.
template <class T, class Op, bool INCL>
__global__ void __launch_bounds__(kScanThreads) scan_tile(T *__restrict__ x, uint64_t n, const T *__restrict__ carry)
{
    constexpr int kItems = scan_items<T>(), kTile = scan_tile_n<T>();
    __shared__ T s[kTile];
    __shared__ T tsum[kScanThreads];
    const int t = threadIdx.x;
    const uint64_t base = (uint64_t)blockIdx.x * kTile;
    for (int j = 0; j < kItems; ++j) {
        const uint64_t i = base + (uint64_t)j * kScanThreads + t;
        s[j * kScanThreads + t] = i < n ? x[i] : Op::id();
    }
    __syncthreads();
    T v[kItems];
    T acc = Op::id();
    for (int j = 0; j < kItems; ++j) {
        v[j] = s[t * kItems + j];
        acc = Op::op(acc, v[j]);
    }
    tsum[t] = acc;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {   // inclusive scan of the thread sums
        const T o = t >= off ? tsum[t - off] : Op::id();
        __syncthreads();
        if (t >= off) tsum[t] = Op::op(o, tsum[t]);
        __syncthreads();
    }
    T run = t ? tsum[t - 1] : Op::id();
    if (carry) run = Op::op(carry[blockIdx.x], run);
    for (int j = 0; j < kItems; ++j) {
        const T in = v[j];
        if (INCL) run = Op::op(run, in);
        s[t * kItems + j] = run;
        if (!INCL) run = Op::op(run, in);
    }
    __syncthreads();
    for (int j = 0; j < kItems; ++j) {
        const uint64_t i = base + (uint64_t)j * kScanThreads + t;
        if (i < n) x[i] = s[j * kScanThreads + t];
    }
}

// Device scratch for the scans' per-tile sums, taken as a stack.
struct Scratch {
    unsigned char *p = nullptr;
    size_t cap = 0, top = 0;
};

template <class T, class Op, bool INCL>
int scan(T *x, uint64_t n, Scratch &scr, cudaStream_t st)
{
    if (n == 0) return 0;
    const uint64_t tiles = (n + scan_tile_n<T>() - 1) / scan_tile_n<T>();
    if (tiles == 1) {
        scan_tile<T, Op, INCL><<<1, kScanThreads, 0, st>>>(x, n, nullptr);
        return cudaGetLastError() == cudaSuccess ? 0 : GALN_ECUDA;
    }
    const size_t bytes = (tiles * sizeof(T) + 255) & ~(size_t)255;
    if (scr.top + bytes > scr.cap) return GALN_ENOMEM;
    T *part = reinterpret_cast<T *>(scr.p + scr.top);
    scr.top += bytes;
    scan_reduce<T, Op><<<(unsigned)tiles, kScanThreads, 0, st>>>(x, n, part);
    int rc = scan<T, Op, false>(part, tiles, scr, st);
    if (!rc) scan_tile<T, Op, INCL><<<(unsigned)tiles, kScanThreads, 0, st>>>(x, n, part);
    scr.top -= bytes;
    if (rc) return rc;
    return cudaGetLastError() == cudaSuccess ? 0 : GALN_ECUDA;
}

// ---- stable LSD radix sort of (uint64 key, V value) pairs, V = uint32 or uint64 positions ----

// counts[d * tiles + tile] = items of digit d in the tile
__global__ void __launch_bounds__(kRThreads) radix_hist(const uint64_t *__restrict__ keys, uint64_t n, int shift,
                                                         uint32_t *__restrict__ counts, uint32_t tiles)
{
    __shared__ uint32_t h[256];
    const int t = threadIdx.x, lane = t & 31;
    if (t < 256) h[t] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kRTile;
    uint32_t dg[kRItems];
#pragma unroll
    for (int j = 0; j < kRItems; ++j) {   // all loads first
        const uint64_t i = base + (uint64_t)j * kRThreads + t;
        dg[j] = i < n ? (uint32_t)(keys[i] >> shift) & 255u : 256u;
    }
#pragma unroll
    for (int j = 0; j < kRItems; ++j) {
        const uint32_t d = dg[j];
        if (__all_sync(0xffffffffu, d == __shfl_sync(0xffffffffu, d, 0))) {   // one digit in the whole warp
            if (lane == 0 && d < 256u) atomicAdd(&h[d], 32u);
            continue;
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (d < 256u && lane == __ffs(peers) - 1) atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    if (t < 256) counts[(uint64_t)t * tiles + blockIdx.x] = h[t];
}

template <class V>
struct ScatterSmem {
    uint32_t wcnt[kRWarps][256];       // per warp: items of each digit, then their offset among the tile's
    uint32_t tstart[256];              // start of each digit in the tile's sorted order
    uint32_t gofs[256];                // the tile's first output index for each digit
    uint32_t wsum[8];
    uint64_t k[kRTile];
    V v[kRTile];
};

// Items of a tile in input order: warp w holds [w * 32 * kRItems, (w + 1) * 32 * kRItems), its step j the
// 32 items from j * 32 on, one per lane. A lane's rank among the warp's items of its digit comes from
// __match_any_sync; warps are ordered by a per-digit prefix over warps; the tile's items are placed in
// digit order in shared memory and leave it in runs.
template <class V>
__global__ void __launch_bounds__(kRThreads) radix_scatter(const uint64_t *__restrict__ kin,
                                                            const V *__restrict__ vin,
                                                            uint64_t *__restrict__ kout, V *__restrict__ vout,
                                                            uint64_t n, int shift, const uint32_t *__restrict__ offsets,
                                                            uint32_t tiles)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScatterSmem<V> &S = *reinterpret_cast<ScatterSmem<V> *>(smem_raw);
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const uint64_t base = (uint64_t)blockIdx.x * kRTile;
    const uint64_t wbase = base + (uint64_t)w * (32 * kRItems);
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint64_t key[kRItems];
    V val[kRItems];
    uint32_t rk[kRItems];
#pragma unroll
    for (int j = 0; j < kRItems; ++j) {   // all loads in flight while the counters are cleared
        const uint64_t i = wbase + (uint64_t)j * 32 + lane;
        const bool ok = i < n;
        key[j] = ok ? kin[i] : 0;
        val[j] = ok ? vin[i] : 0;
    }
    for (int i = t; i < kRWarps * 256; i += kRThreads) (&S.wcnt[0][0])[i] = 0;
    if (t < 256) S.gofs[t] = offsets[(uint64_t)t * tiles + blockIdx.x];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kRItems; ++j) {
        const bool ok = wbase + (uint64_t)j * 32 + lane < n;
        const uint32_t d = ok ? (uint32_t)(key[j] >> shift) & 255u : 256u;
        const bool uni = __all_sync(0xffffffffu, d == __shfl_sync(0xffffffffu, d, 0));
        const uint32_t peers = uni ? 0xffffffffu : __match_any_sync(0xffffffffu, d);
        const uint32_t c = ok ? S.wcnt[w][d] : 0u;
        rk[j] = c + (uint32_t)__popc(peers & lt_mask);
        __syncwarp();
        if (ok && (peers & lt_mask) == 0) S.wcnt[w][d] = c + (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    uint32_t tot = 0;
    if (t < 256) {
        for (int ww = 0; ww < kRWarps; ++ww) {
            const uint32_t c = S.wcnt[ww][t];
            S.wcnt[ww][t] = tot;
            tot += c;
        }
    }
    // exclusive scan of the 256 digit totals (threads 0..255 = warps 0..7)
    uint32_t inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (t < 256 && lane == 31) S.wsum[w] = inc;
    __syncthreads();
    if (t < 256) {
        uint32_t before = 0;
        for (int ww = 0; ww < w; ++ww) before += S.wsum[ww];
        S.tstart[t] = before + inc - tot;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kRItems; ++j) {
        const uint64_t i = wbase + (uint64_t)j * 32 + lane;
        if (i < n) {
            const uint32_t d = (uint32_t)(key[j] >> shift) & 255u;
            const uint32_t p = S.tstart[d] + S.wcnt[w][d] + rk[j];
            S.k[p] = key[j];
            S.v[p] = val[j];
        }
    }
    __syncthreads();
    const uint32_t tile_n = (uint32_t)min((uint64_t)kRTile, n - base);
    for (uint32_t i = t; i < tile_n; i += kRThreads) {
        const uint64_t kk = S.k[i];
        const uint32_t d = (uint32_t)(kk >> shift) & 255u;
        const uint64_t dst = (uint64_t)S.gofs[d] + (i - S.tstart[d]);
        kout[dst] = kk;
        vout[dst] = S.v[i];
    }
}

template <class V>
struct Sorter {
    uint64_t *k[2] = {nullptr, nullptr};
    V *v[2] = {nullptr, nullptr};
    uint32_t *counts = nullptr;
    Scratch *scr = nullptr;
    int passes = 0;
    uint64_t scatter_items = 0;
    std::vector<cudaEvent_t> ev;       // start/stop pairs around each scatter launch
};

// Sorts the n pairs in (k[cur], v[cur]) on key bits [0, bits); returns the buffer that holds them sorted.
template <class V>
int radix_sort(Sorter<V> &s, int cur, uint64_t n, int bits, cudaStream_t st, int &out)
{
    out = cur;
    if (n <= 1) return 0;
    const uint32_t tiles = (uint32_t)((n + kRTile - 1) / kRTile);
    for (int shift = 0; shift < bits; shift += 8) {
        radix_hist<<<tiles, kRThreads, 0, st>>>(s.k[cur], n, shift, s.counts, tiles);
        int rc = scan<uint32_t, OpSum<uint32_t>, false>(s.counts, (uint64_t)tiles * 256, *s.scr, st);
        if (rc) return rc;
        cudaEvent_t a, b;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return GALN_ECUDA;
        s.ev.push_back(a);
        s.ev.push_back(b);
        cudaEventRecord(a, st);
        radix_scatter<V><<<tiles, kRThreads, sizeof(ScatterSmem<V>), st>>>(s.k[cur], s.v[cur], s.k[cur ^ 1],
                                                                           s.v[cur ^ 1], n, shift, s.counts, tiles);
        cudaEventRecord(b, st);
        if (cudaGetLastError() != cudaSuccess) return GALN_ECUDA;
        cur ^= 1;
        ++s.passes;
        s.scatter_items += n;
    }
    out = cur;
    return 0;
}

// ---- prefix doubling ----

__global__ void pd_key0(const uint8_t *__restrict__ T, uint64_t N, uint64_t *__restrict__ key, uint32_t *__restrict__ pos)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    uint64_t k = 0;
    for (int j = 0; j < kPrefix; ++j) {
        const uint64_t p = i + j;
        k = (k << 3) | (p < N ? (uint64_t)T[p] + 1 : 0);
    }
    key[i] = k;
    pos[i] = (uint32_t)i;
}

// H[k] = the slot of item k if it starts a group of equal keys, else 0 (an inclusive max-scan then gives
// every item its group's first slot). Slots rise with k; round 0's slot of item k is k.
__global__ void pd_heads(const uint64_t *__restrict__ K, const uint32_t *__restrict__ slot, uint64_t M,
                         uint32_t *__restrict__ H)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const bool head = k == 0 || K[k] != K[k - 1];
    H[k] = head ? (slot ? slot[k] : (uint32_t)k) : 0u;
}

// rank[position] = its group's first slot; C[k] = 1 when item k stays unsorted (its group has two or more)
__global__ void pd_rank(const uint64_t *__restrict__ K, const uint32_t *__restrict__ P, const uint32_t *__restrict__ H,
                        uint64_t M, uint32_t *__restrict__ rank, uint32_t *__restrict__ C)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const bool head = k == 0 || K[k] != K[k - 1];
    const bool last = k + 1 == M || K[k + 1] != K[k];
    rank[P[k]] = H[k];
    C[k] = (head && last) ? 0u : 1u;
}

// C: inclusive count of kept items. Kept item k goes to C[k] - 1 with its position and slot.
__global__ void pd_compact(const uint32_t *__restrict__ P, const uint32_t *__restrict__ slot,
                           const uint32_t *__restrict__ C, uint64_t M, uint32_t *__restrict__ P2,
                           uint32_t *__restrict__ slot2)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const uint32_t c = C[k], prev = k ? C[k - 1] : 0u;
    if (c == prev) return;
    P2[c - 1] = P[k];
    slot2[c - 1] = slot ? slot[k] : (uint32_t)k;
}

// key of an unsorted suffix p: (rank of p, rank of p + h plus one; 0 when p + h is the end of the text)
__global__ void pd_key(const uint32_t *__restrict__ P, const uint32_t *__restrict__ rank, uint64_t M, uint64_t N,
                       uint64_t h, int lo_bits, uint64_t *__restrict__ K)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const uint64_t p = P[k], q = p + h;
    const uint64_t lo = q < N ? (uint64_t)rank[q] + 1 : 0;
    K[k] = ((uint64_t)rank[p] << lo_bits) | lo;
}

__global__ void pd_sa(const uint32_t *__restrict__ rank, uint64_t N, uint32_t *__restrict__ sa)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) sa[(uint64_t)rank[i] + 1] = (uint32_t)i;
    if (i == 0) sa[0] = (uint32_t)N;
}

// ---- BWT, .bwt body, .sa samples ----

// L[s], s = 0..N-1: the BWT of T$ without the $ of row `primary`; row 0 (the $ suffix) gives T[N-1]
__global__ void bwt_symbols(const uint8_t *__restrict__ T, const uint32_t *__restrict__ sa, uint64_t N, uint64_t primary,
                            uint8_t *__restrict__ L)
{
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const uint64_t row = s < primary ? s : s + 1;
    L[s] = T[(uint64_t)sa[row] - 1];
}

__global__ void bwt_block_counts(const uint8_t *__restrict__ L, uint64_t N, uint64_t nb, U4 *__restrict__ cnt)
{
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint64_t s = b * 128, e = min(s + 128, N);
    uint64_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    for (uint64_t i = s; i < e; ++i) {
        const uint8_t x = L[i];
        c0 += x == 0; c1 += x == 1; c2 += x == 2; c3 += x == 3;
    }
    cnt[b] = U4{{c0, c1, c2, c3}};
}

// 16 words per 128-symbol block: the four uint64 counts before it, then 8 words of 16 symbols, the first
// symbol in the top two bits. incl = inclusive per-block counts. Words past the text are not written.
__global__ void bwt_write(const uint8_t *__restrict__ L, uint64_t N, uint64_t nb, const U4 *__restrict__ incl,
                          uint32_t *__restrict__ body)
{
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nb * 16) return;
    const uint64_t b = idx >> 4;
    const int j = (int)(idx & 15);
    if (j < 8) {
        const uint64_t v = b ? incl[b - 1].c[j >> 1] : 0;
        body[idx] = (j & 1) ? (uint32_t)(v >> 32) : (uint32_t)v;
        return;
    }
    const uint64_t s0 = b * 128 + (uint64_t)(j - 8) * 16;
    if (s0 >= N) return;
    uint32_t word = 0;
    for (int t = 0; t < 16; ++t)
        if (s0 + t < N) word |= (uint32_t)L[s0 + t] << (30 - 2 * t);
    body[idx] = word;
}

__global__ void sa_samples(const uint32_t *__restrict__ sa, uint64_t ns, uint64_t *__restrict__ out)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < ns) out[k] = sa[(k + 1) * 32];
}

__global__ void text_from_forward(const uint8_t *__restrict__ F, uint64_t l_pac, uint8_t *__restrict__ T)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * l_pac) return;
    T[i] = i < l_pac ? F[i] : (uint8_t)(3 - F[2 * l_pac - 1 - i]);
}

inline unsigned grid(uint64_t n, int b) { return (unsigned)((n + b - 1) / b); }
inline int bitlen(uint64_t x) { return x ? 64 - __builtin_clzll(x) : 0; }

// ---- the 64-bit path (texts of 2^32 - 64 symbols or more) ----
// Positions, ranks and slots are 64-bit. Round 0 runs bucket by bucket: suffixes are grouped by their first
// kWPre symbols (a histogram of those prefix codes, then runs of consecutive codes holding at most `chunk`
// suffixes), each bucket's suffixes are selected from the text, sorted by their 21-symbol keys and ranked;
// the unsorted ones are appended to one list U of (position, slot) in slot order. A later round walks U in
// chunks of whole groups: each item's key is (its group's number in the chunk, rank of p + h), the chunk is
// sorted, ranked and its still-unsorted items compacted back into U in place. Ranks are updated while the
// round goes on: a rank that another chunk has refined already is still consistent with the suffix order
// (its group only split into ordered parts), so sorting by it can only refine further (Larsson-Sadakane's
// argument). The BWT and the SA samples are scattered from the final ranks without a suffix array.
constexpr int kWPre = 5;                                  // symbols of a bucket prefix
constexpr uint32_t kWCodes = 1u << (3 * kWPre);           // prefix codes (3 bits a symbol)
constexpr int kWHistTile = 1 << 20;                       // text positions per histogram block
constexpr int kWSelTile = 1 << 14;                        // text positions per selection block
constexpr int kWSelThreads = 256;

__device__ __forceinline__ uint64_t key21(const uint8_t *__restrict__ T, uint64_t N, uint64_t i)
{
    uint64_t k = 0;
    for (int j = 0; j < kPrefix; ++j) {
        const uint64_t p = i + j;
        k = (k << 3) | (p < N ? (uint64_t)T[p] + 1 : 0);
    }
    return k;
}

__device__ __forceinline__ uint32_t code5(const uint8_t *__restrict__ T, uint64_t N, uint64_t i)
{
    uint32_t c = 0;
    for (int j = 0; j < kWPre; ++j) {
        const uint64_t p = i + j;
        c = (c << 3) | (p < N ? (uint32_t)T[p] + 1 : 0u);
    }
    return c;
}

// hist[c] += the text positions whose kWPre-symbol prefix code is c (a shared-memory histogram per block)
__global__ void __launch_bounds__(1024) w_hist(const uint8_t *__restrict__ T, uint64_t N,
                                               unsigned long long *__restrict__ hist)
{
    extern __shared__ uint32_t hs[];
    for (uint32_t c = threadIdx.x; c < kWCodes; c += blockDim.x) hs[c] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kWHistTile;
    const uint64_t end = min(N, base + kWHistTile);
    for (uint64_t i = base + threadIdx.x; i < end; i += blockDim.x) atomicAdd(&hs[code5(T, N, i)], 1u);
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < kWCodes; c += blockDim.x)
        if (hs[c]) atomicAdd(&hist[c], (unsigned long long)hs[c]);
}

// per selection tile: how many positions have a prefix code in [lo, hi]
__global__ void __launch_bounds__(kWSelThreads) w_sel_count(const uint8_t *__restrict__ T, uint64_t N, uint32_t lo,
                                                            uint32_t hi, uint32_t *__restrict__ tcount)
{
    __shared__ uint32_t s[kWSelThreads / 32];
    const uint64_t base = (uint64_t)blockIdx.x * kWSelTile;
    const uint64_t end = min(N, base + kWSelTile);
    uint32_t c = 0;
    for (uint64_t i = base + threadIdx.x; i < end; i += kWSelThreads) {
        const uint32_t x = code5(T, N, i);
        c += (x >= lo && x <= hi) ? 1u : 0u;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kWSelThreads / 32; ++w) t += s[w];
        tcount[blockIdx.x] = t;
    }
}

// writes the selected positions in text order (tile offsets from an exclusive scan of w_sel_count) with
// their 21-symbol keys
__global__ void __launch_bounds__(kWSelThreads) w_sel_write(const uint8_t *__restrict__ T, uint64_t N, uint32_t lo,
                                                            uint32_t hi, const uint32_t *__restrict__ toff,
                                                            uint64_t *__restrict__ K, uint64_t *__restrict__ P)
{
    __shared__ uint32_t s[kWSelThreads / 32];
    __shared__ uint32_t run;
    const uint64_t base = (uint64_t)blockIdx.x * kWSelTile;
    const uint64_t end = min(N, base + kWSelTile);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) run = toff[blockIdx.x];
    __syncthreads();
    for (uint64_t i0 = base; i0 < end; i0 += kWSelThreads) {
        const uint64_t i = i0 + threadIdx.x;
        const uint32_t x = i < end ? code5(T, N, i) : 0u;
        const bool sel = i < end && x >= lo && x <= hi;
        const uint32_t b = __ballot_sync(0xffffffffu, sel);
        if (lane == 0) s[w] = (uint32_t)__popc(b);
        __syncthreads();
        uint32_t before = run;
        for (int ww = 0; ww < w; ++ww) before += s[ww];
        if (sel) {
            const uint64_t o = before + (uint32_t)__popc(b & ((1u << lane) - 1u));
            K[o] = key21(T, N, i);
            P[o] = i;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int ww = 0; ww < kWSelThreads / 32; ++ww) t += s[ww];
            run += t;
        }
        __syncthreads();
    }
}

// H[k] = slot of item k (slot0 + k, or slot[k]) if its key starts a group, else 0
__global__ void w_heads(const uint64_t *__restrict__ K, uint64_t M, uint64_t slot0, const uint64_t *__restrict__ slot,
                        uint64_t *__restrict__ H)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const bool head = k == 0 || K[k] != K[k - 1];
    H[k] = head ? (slot ? slot[k] : slot0 + k) : 0;
}

// rank[position] = its group's first slot; C[k] = 1 when item k stays unsorted
__global__ void w_rank(const uint64_t *__restrict__ K, const uint64_t *__restrict__ P, const uint64_t *__restrict__ H,
                       uint64_t M, uint64_t *__restrict__ rank, uint32_t *__restrict__ C)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const bool head = k == 0 || K[k] != K[k - 1];
    const bool last = k + 1 == M || K[k + 1] != K[k];
    rank[P[k]] = H[k];
    C[k] = (head && last) ? 0u : 1u;
}

// kept item k goes to U at out + C[k] - 1 with its position and slot (slot0 + k, or slot[k])
__global__ void w_compact(const uint64_t *__restrict__ P, const uint32_t *__restrict__ C, uint64_t M, uint64_t slot0,
                          const uint64_t *__restrict__ slot, uint64_t out, uint64_t *__restrict__ Upos,
                          uint64_t *__restrict__ Uslot)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const uint32_t c = C[k], prev = k ? C[k - 1] : 0u;
    if (c == prev) return;
    Upos[out + c - 1] = P[k];
    Uslot[out + c - 1] = slot ? slot[k] : slot0 + k;
}

// group starts of U's items [a, a + m): F[k] = 1 when item a + k starts a group (its rank differs from the
// item before it); the flags' inclusive scan numbers the groups
__global__ void w_group_flags(const uint64_t *__restrict__ Upos, uint64_t a, uint64_t m, const uint64_t *__restrict__ rank,
                              uint32_t *__restrict__ F)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    F[k] = (k == 0 || rank[Upos[a + k]] != rank[Upos[a + k - 1]]) ? 1u : 0u;
}

// the last group start in U's items (a, e], or a when there is none (one group fills the window)
__global__ void w_last_start(const uint64_t *__restrict__ Upos, uint64_t a, uint64_t e, const uint64_t *__restrict__ rank,
                             unsigned long long *__restrict__ best)
{
    const uint64_t k = a + 1 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k > e) return;
    if (rank[Upos[k]] != rank[Upos[k - 1]]) atomicMax(best, (unsigned long long)k);
}

// key of chunk item k: (its group number, rank of p + h plus one; 0 past the end), position as the value;
// the chunk's slots are copied aside (U's slot array is overwritten by the compaction)
__global__ void w_key(const uint64_t *__restrict__ Upos, const uint64_t *__restrict__ Uslot, uint64_t a, uint64_t m,
                      const uint32_t *__restrict__ G, const uint64_t *__restrict__ rank, uint64_t N, uint64_t h,
                      int lo_bits, uint64_t *__restrict__ K, uint64_t *__restrict__ P)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const uint64_t p = Upos[a + k], q = p + h;
    const uint64_t lo = q < N ? rank[q] + 1 : 0;
    K[k] = ((uint64_t)(G[k] - 1) << lo_bits) | lo;
    P[k] = p;
}

__global__ void w_copy_u64(const uint64_t *__restrict__ src, uint64_t m, uint64_t *__restrict__ dst)
{
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) dst[k] = src[k];
}

// the BWT without the $ of row `primary` (row r's symbol is T[SA[r] - 1]; suffix i is at row rank[i] + 1,
// the $ suffix at row 0) and the SA samples of rows 32, 64, ...
__global__ void w_bwt_scatter(const uint8_t *__restrict__ T, const uint64_t *__restrict__ rank, uint64_t N,
                              uint64_t primary, uint8_t *__restrict__ L, uint64_t *__restrict__ smp)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (i == 0) L[0] = T[N - 1];
    const uint64_t row = rank[i] + 1;
    if (i > 0) L[row < primary ? row : row - 1] = T[i - 1];
    if ((row & 31) == 0) smp[row / 32 - 1] = i;
}

struct DevMem {
    std::vector<void *> ptrs;
    ~DevMem()
    {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    T *get(size_t count)
    {
        void *p = nullptr;
        if (cudaMalloc(&p, std::max<size_t>(count * sizeof(T), 256)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
};

// Round 0 of the 64-bit path, then the doubling rounds over U; fills rank[0..N). Returns 0 or an error.
int wide_sort(const uint8_t *T, uint64_t N, uint64_t *rank, Sorter<uint64_t> &srt, Scratch &scr, uint64_t chunk,
              uint64_t *Upos, uint64_t *Uslot, uint64_t ucap, uint32_t *tcount, unsigned long long *hist,
              unsigned long long *best, cudaStream_t st, int &rounds, uint64_t &sorted)
{
    rounds = 0;
    sorted = 0;
    // bucket plan: runs of consecutive prefix codes holding at most `chunk` suffixes each
    if (cudaMemsetAsync(hist, 0, kWCodes * 8, st) != cudaSuccess) return GALN_ECUDA;
    w_hist<<<grid(N, kWHistTile), 1024, kWCodes * 4, st>>>(T, N, hist);
    std::vector<unsigned long long> h(kWCodes);
    if (cudaMemcpyAsync(h.data(), hist, kWCodes * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return GALN_ECUDA;
    const uint64_t sel_tiles = (N + kWSelTile - 1) / kWSelTile;
    uint64_t u_n = 0, slot0 = 0;
    uint32_t lo = 0;
    while (lo < kWCodes) {
        uint64_t m = 0;
        uint32_t hi = lo;
        while (hi < kWCodes && (m + h[hi] <= chunk || (m == 0 && h[hi] <= chunk))) m += h[hi++];
        if (hi == lo) {
            fprintf(stderr, "[galn index] %llu suffixes share a %d-symbol prefix: more than %llu at once\n",
                    (unsigned long long)h[lo], kWPre, (unsigned long long)chunk);
            return GALN_ENOMEM;
        }
        if (m > 0) {
            w_sel_count<<<(unsigned)sel_tiles, kWSelThreads, 0, st>>>(T, N, lo, hi - 1, tcount);
            int rc = scan<uint32_t, OpSum<uint32_t>, false>(tcount, sel_tiles, scr, st);
            if (rc) return rc;
            w_sel_write<<<(unsigned)sel_tiles, kWSelThreads, 0, st>>>(T, N, lo, hi - 1, tcount, srt.k[0], srt.v[0]);
            int kb = 0;
            rc = radix_sort(srt, 0, m, 3 * kPrefix, st, kb);
            if (rc) return rc;
            sorted += m;
            uint64_t *H = srt.k[kb ^ 1];
            uint32_t *C = reinterpret_cast<uint32_t *>(srt.v[kb ^ 1]);
            w_heads<<<grid(m, 256), 256, 0, st>>>(srt.k[kb], m, slot0, nullptr, H);
            rc = scan<uint64_t, OpMax<uint64_t>, true>(H, m, scr, st);
            if (rc) return rc;
            w_rank<<<grid(m, 256), 256, 0, st>>>(srt.k[kb], srt.v[kb], H, m, rank, C);
            rc = scan<uint32_t, OpSum<uint32_t>, true>(C, m, scr, st);
            if (rc) return rc;
            uint32_t kept = 0;
            if (cudaMemcpyAsync(&kept, C + m - 1, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return GALN_ECUDA;
            if (u_n + kept > ucap) {
                fprintf(stderr, "[galn index] %llu unsorted suffixes after the first sort: more than fit\n",
                        (unsigned long long)(u_n + kept));
                return GALN_ENOMEM;
            }
            w_compact<<<grid(m, 256), 256, 0, st>>>(srt.v[kb], C, m, slot0, nullptr, u_n, Upos, Uslot);
            u_n += kept;
            slot0 += m;
        }
        lo = hi;
    }
    if (slot0 != N) return GALN_ECUDA;
    // doubling rounds over U in chunks of whole groups
    const int lo_bits = bitlen(N);
    uint64_t h2 = kPrefix;
    while (u_n > 0) {
        if (++rounds > kMaxRounds) return GALN_EINVAL;
        uint64_t a = 0, out = 0;
        while (a < u_n) {
            uint64_t e = std::min(u_n, a + chunk);
            if (e < u_n) {   // end the chunk at the last group start inside the window
                unsigned long long b = a;
                if (cudaMemcpyAsync(best, &b, 8, cudaMemcpyHostToDevice, st) != cudaSuccess) return GALN_ECUDA;
                w_last_start<<<grid(e - a, 256), 256, 0, st>>>(Upos, a, e, rank, best);
                if (cudaMemcpyAsync(&b, best, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess)
                    return GALN_ECUDA;
                if (b == a) {
                    fprintf(stderr, "[galn index] a group of more than %llu suffixes\n", (unsigned long long)chunk);
                    return GALN_ENOMEM;
                }
                e = b;
            }
            const uint64_t m = e - a;
            uint32_t *G = reinterpret_cast<uint32_t *>(srt.k[1]);
            w_group_flags<<<grid(m, 256), 256, 0, st>>>(Upos, a, m, rank, G);
            int rc = scan<uint32_t, OpSum<uint32_t>, true>(G, m, scr, st);
            if (rc) return rc;
            uint32_t n_groups = 0;
            if (cudaMemcpyAsync(&n_groups, G + m - 1, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return GALN_ECUDA;
            if (bitlen(n_groups) + lo_bits > 64) return GALN_EINVAL;
            w_key<<<grid(m, 256), 256, 0, st>>>(Upos, Uslot, a, m, G, rank, N, h2, lo_bits, srt.k[0], srt.v[0]);
            int kb = 0;
            rc = radix_sort(srt, 0, m, lo_bits + bitlen(n_groups - 1), st, kb);
            if (rc) return rc;
            sorted += m;
            uint64_t *H = srt.k[kb ^ 1];
            uint32_t *C = reinterpret_cast<uint32_t *>(srt.v[kb ^ 1]);
            w_heads<<<grid(m, 256), 256, 0, st>>>(srt.k[kb], m, 0, Uslot + a, H);
            rc = scan<uint64_t, OpMax<uint64_t>, true>(H, m, scr, st);
            if (rc) return rc;
            w_rank<<<grid(m, 256), 256, 0, st>>>(srt.k[kb], srt.v[kb], H, m, rank, C);
            rc = scan<uint32_t, OpSum<uint32_t>, true>(C, m, scr, st);
            if (rc) return rc;
            uint32_t kept = 0;
            if (cudaMemcpyAsync(&kept, C + m - 1, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                return GALN_ECUDA;
            // the chunk's slots aside (H is consumed), then compacted into U in place: every write lands at
            // or before the chunk's own start
            w_copy_u64<<<grid(m, 256), 256, 0, st>>>(Uslot + a, m, H);
            w_compact<<<grid(m, 256), 256, 0, st>>>(srt.v[kb], C, m, 0, H, out, Upos, Uslot);
            out += kept;
            a = e;
        }
        u_n = out;
        h2 *= 2;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : GALN_ECUDA;
}

}  // namespace ixb

// The 64-bit device part (see the 64-bit path above): forward sequence (host) -> .bwt words, L2, primary,
// .sa samples (host). chunk: suffixes sorted at once (0: from free device memory).
static int dev_build_bwt_sa_wide(const uint8_t *F, uint64_t l_pac, std::vector<uint32_t> &bwt, uint64_t L2[5],
                                 uint64_t &primary, std::vector<uint64_t> &samples, galn_build_stats *stats,
                                 uint64_t chunk)
{
    using namespace ixb;
    const uint64_t N = 2 * l_pac;
    if (l_pac == 0 || N >= (1ull << 40)) return GALN_EINVAL;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return GALN_ECUDA;
    // fixed: text, ranks, bucket histogram, selection tile counts; per sorted suffix 32 bytes (keys, values)
    // plus radix tile counts; U: 16 bytes per unsorted suffix; the end: BWT bytes, block counts and body
    const uint64_t sel_tiles = (N + kWSelTile - 1) / kWSelTile;
    const size_t fixed = (size_t)N + 64 + (size_t)N * 8 + kWCodes * 8 + sel_tiles * 4 + (256ull << 20);
    if (!chunk) {
        const size_t spare = fr > fixed ? fr - fixed : 0;
        chunk = std::min<uint64_t>(N, std::max<uint64_t>(1 << 20, spare / 4 / 34));   // a quarter for sorting
        chunk = std::min<uint64_t>(chunk, 1ull << 31);
    }
    chunk = std::min<uint64_t>(chunk, N);
    const uint64_t rtiles = (chunk + kRTile - 1) / kRTile;
    const size_t sort_bytes = (size_t)chunk * 32 + rtiles * 1024 + (size_t)(chunk / 1000 + 4096) * 32;
    if (fixed + sort_bytes + (16ull << 20) > fr) {
        fprintf(stderr, "[galn index] a text of %llu symbols needs more than %.1f GB of device memory, %.1f GB free\n",
                (unsigned long long)N, (fixed + sort_bytes) / 1e9, fr / 1e9);
        return GALN_ENOMEM;
    }
    const uint64_t ucap = std::min<uint64_t>(N, (fr - fixed - sort_bytes - (16ull << 20)) / 16);
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return GALN_ECUDA;
    cudaFuncSetAttribute(radix_scatter<uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(ScatterSmem<uint64_t>));
    cudaFuncSetAttribute(w_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kWCodes * 4));
    const uint64_t nb = (N + 127) / 128, nw = (N + 15) / 16;
    const uint64_t body_words = 16 * nb - (8 - (nw - 8 * (nb - 1)));
    const uint64_t ns = (N + 32) / 32 - 1;
    bwt.resize(body_words + 8);
    samples.resize(ns);
    int rc = 0;
    cudaEvent_t ea, e0, e1, eb;
    cudaEventCreate(&ea);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&eb);
    Sorter<uint64_t> srt;
    Scratch scr;
    int rounds = 0;
    uint64_t sorted = 0;
    {
        DevMem m;
        uint8_t *T = m.get<uint8_t>(N + 64);
        uint64_t *rank = m.get<uint64_t>(N);
        unsigned long long *hist = m.get<unsigned long long>(kWCodes + 1);
        uint32_t *tcount = m.get<uint32_t>(sel_tiles);
        if (!T || !rank || !hist || !tcount) rc = GALN_ENOMEM;
        if (!rc) {
            cudaEventRecord(ea, st);
            // the forward half and its reverse complement, uploaded through the end of T (freed after)
            DevMem fm;
            uint8_t *F_d = fm.get<uint8_t>(l_pac);
            if (!F_d) rc = GALN_ENOMEM;
            if (!rc) {
                cudaMemcpyAsync(F_d, F, l_pac, cudaMemcpyHostToDevice, st);
                cudaEventRecord(e0, st);
                text_from_forward<<<grid(N, 256), 256, 0, st>>>(F_d, l_pac, T);
                cudaMemsetAsync(T + N, 0, 64, st);
                if (cudaStreamSynchronize(st) != cudaSuccess) rc = GALN_ECUDA;
            }
        }
        if (!rc) {
            DevMem sm;
            srt.k[0] = sm.get<uint64_t>(chunk);
            srt.k[1] = sm.get<uint64_t>(chunk);
            srt.v[0] = sm.get<uint64_t>(chunk);
            srt.v[1] = sm.get<uint64_t>(chunk);
            srt.counts = sm.get<uint32_t>(rtiles * 256);
            scr.cap = (size_t)(chunk / 1000 + 4096) * 32;
            scr.p = sm.get<unsigned char>(scr.cap);
            srt.scr = &scr;
            uint64_t *Upos = sm.get<uint64_t>(ucap), *Uslot = sm.get<uint64_t>(ucap);
            if (!srt.k[0] || !srt.k[1] || !srt.v[0] || !srt.v[1] || !srt.counts || !scr.p || !Upos || !Uslot)
                rc = GALN_ENOMEM;
            if (!rc) rc = wide_sort(T, N, rank, srt, scr, chunk, Upos, Uslot, ucap, tcount, hist, hist + kWCodes, st,
                                    rounds, sorted);
            if (rc) cudaStreamSynchronize(st);
        }
        if (!rc) {
            uint64_t r0 = 0;
            if (cudaMemcpyAsync(&r0, rank, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                rc = GALN_ECUDA;
            primary = r0 + 1;
        }
        if (!rc) {
            DevMem em;
            uint8_t *L = em.get<uint8_t>(N);
            U4 *cnt = em.get<U4>(nb);
            uint32_t *body = em.get<uint32_t>(nb * 16);
            uint64_t *smp = em.get<uint64_t>(std::max<uint64_t>(ns, 1));
            scr.cap = (size_t)(nb / 100 + 4096) * 64;
            scr.top = 0;
            scr.p = em.get<unsigned char>(scr.cap);
            if (!L || !cnt || !body || !smp || !scr.p) rc = GALN_ENOMEM;
            if (!rc) {
                w_bwt_scatter<<<grid(N, 256), 256, 0, st>>>(T, rank, N, primary, L, smp);
                bwt_block_counts<<<grid(nb, 128), 128, 0, st>>>(L, N, nb, cnt);
                rc = scan<U4, OpSum<U4>, true>(cnt, nb, scr, st);
            }
            if (!rc) {
                bwt_write<<<grid(nb * 16, 256), 256, 0, st>>>(L, N, nb, cnt, body);
                U4 totals{};
                cudaEventRecord(e1, st);
                cudaMemcpyAsync(bwt.data(), body, body_words * 4, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(&totals, cnt + nb - 1, sizeof(U4), cudaMemcpyDeviceToHost, st);
                if (ns) cudaMemcpyAsync(samples.data(), smp, ns * 8, cudaMemcpyDeviceToHost, st);
                cudaEventRecord(eb, st);
                if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = GALN_ECUDA;
                if (!rc) {
                    memcpy(bwt.data() + body_words, totals.c, sizeof(totals.c));
                    L2[0] = 0;
                    for (int c = 0; c < 4; ++c) L2[c + 1] = L2[c] + totals.c[c];
                }
            }
            if (rc) cudaStreamSynchronize(st);
        }
        if (stats && !rc) {
            stats->n = N;
            stats->primary = primary;
            stats->rounds = rounds;
            stats->sorted_items = sorted;
            stats->sort_passes = srt.passes;
            stats->scatter_items = srt.scatter_items;
            float ms = 0, up = 0, down = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            cudaEventElapsedTime(&up, ea, e0);
            cudaEventElapsedTime(&down, e1, eb);
            stats->ms_device = ms;
            stats->ms_copies = up + down;
            double sc = 0;
            for (size_t i = 0; i + 1 < srt.ev.size(); i += 2) {
                float x = 0;
                cudaEventElapsedTime(&x, srt.ev[i], srt.ev[i + 1]);
                sc += x;
            }
            stats->ms_scatter = sc;
        }
    }
    for (cudaEvent_t e : srt.ev) cudaEventDestroy(e);
    cudaEventDestroy(ea);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(eb);
    cudaStreamDestroy(st);
    if (rc == GALN_ECUDA) cudaGetLastError();
    return rc;
}

// The whole device part: forward sequence (host) -> .bwt words, L2, primary, .sa samples (host). Texts of
// 2^32 - 64 symbols or more, or any text when sort_chunk > 0, take the 64-bit path.
int dev_build_bwt_sa(const uint8_t *F, uint64_t l_pac, std::vector<uint32_t> &bwt, uint64_t L2[5], uint64_t &primary,
                     std::vector<uint64_t> &samples, galn_build_stats *stats, int64_t sort_chunk)
{
    using namespace ixb;
    const uint64_t N = 2 * l_pac;
    if (sort_chunk > 0 || (l_pac > 0 && N > 0xFFFFFFFFull - 64))
        return dev_build_bwt_sa_wide(F, l_pac, bwt, L2, primary, samples, stats,
                                     sort_chunk > 0 ? (uint64_t)sort_chunk : 0);
    if (l_pac == 0) return GALN_EINVAL;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return GALN_ECUDA;
    const uint64_t tiles = (N + kRTile - 1) / kRTile;
    const size_t need = (size_t)N * 38 + tiles * 1024 + (64ull << 20);
    if (need > fr) {
        fprintf(stderr, "[galn index] a text of %llu symbols needs about %.1f GB of device memory, %.1f GB free\n",
                (unsigned long long)N, need / 1e9, fr / 1e9);
        return GALN_ENOMEM;
    }
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return GALN_ECUDA;
    // per device: the attribute belongs to the current device's context
    cudaFuncSetAttribute(radix_scatter<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(ScatterSmem<uint32_t>));
    // the copies go straight from and to the caller's pageable arrays: page-locking them for one build costs
    // more host time than the copies save
    const uint64_t nb = (N + 127) / 128, nw = (N + 15) / 16;
    const uint64_t body_words = 16 * nb - (8 - (nw - 8 * (nb - 1)));
    const uint64_t ns = (N + 32) / 32 - 1;
    bwt.resize(body_words + 8);
    samples.resize(ns);
    int rc = 0;
    cudaEvent_t ea, e0, e1, eb;   // upload start, text in HBM, results in HBM, results on the host
    cudaEventCreate(&ea);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&eb);
    Sorter<uint32_t> srt;
    Scratch scr;
    {
        DevMem m;
        uint8_t *F_d = m.get<uint8_t>(l_pac);
        uint8_t *T = m.get<uint8_t>(N + 64);
        uint32_t *rank = m.get<uint32_t>(N + 1);
        srt.k[0] = m.get<uint64_t>(N);
        srt.k[1] = m.get<uint64_t>(N);
        srt.v[0] = m.get<uint32_t>(N);
        srt.v[1] = m.get<uint32_t>(N);
        uint32_t *slots[2] = {m.get<uint32_t>(N), m.get<uint32_t>(N)};
        srt.counts = m.get<uint32_t>(tiles * 256);
        scr.cap = (size_t)(N / 1000 + 4096) * 32;
        scr.p = m.get<unsigned char>(scr.cap);
        srt.scr = &scr;
        if (!F_d || !T || !rank || !srt.k[0] || !srt.k[1] || !srt.v[0] || !srt.v[1] || !slots[0] || !slots[1] ||
            !srt.counts || !scr.p) {
            rc = GALN_ENOMEM;
        }
        if (!rc) {
            cudaEventRecord(ea, st);
            cudaMemcpyAsync(F_d, F, l_pac, cudaMemcpyHostToDevice, st);
            cudaEventRecord(e0, st);
            text_from_forward<<<grid(N, 256), 256, 0, st>>>(F_d, l_pac, T);
            cudaMemsetAsync(T + N, 0, 64, st);
            pd_key0<<<grid(N, 256), 256, 0, st>>>(T, N, srt.k[0], srt.v[0]);
        }
        // round 0 over all N suffixes; later rounds over the unsorted ones (positions P, slots S)
        int kb = 0, sbuf = 0;
        uint64_t M = N, h = kPrefix;
        const uint32_t *S = nullptr;
        int bits = 3 * kPrefix;
        int rounds = 0;
        uint64_t sorted = 0;
        while (!rc) {
            rc = radix_sort(srt, kb, M, bits, st, kb);
            if (rc) break;
            sorted += M;
            const uint64_t *K = srt.k[kb];
            const uint32_t *P = srt.v[kb];
            // the other key buffer is free: two uint32 arrays of M
            uint32_t *H = reinterpret_cast<uint32_t *>(srt.k[kb ^ 1]);
            uint32_t *C = H + M;
            pd_heads<<<grid(M, 256), 256, 0, st>>>(K, S, M, H);
            rc = scan<uint32_t, OpMax<uint32_t>, true>(H, M, scr, st);
            if (rc) break;
            pd_rank<<<grid(M, 256), 256, 0, st>>>(K, P, H, M, rank, C);
            rc = scan<uint32_t, OpSum<uint32_t>, true>(C, M, scr, st);
            if (rc) break;
            uint32_t kept = 0;
            if (cudaMemcpyAsync(&kept, C + M - 1, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                rc = GALN_ECUDA;
                break;
            }
            if (kept == 0) break;
            if (++rounds > kMaxRounds) { rc = GALN_EINVAL; break; }
            uint32_t *P2 = srt.v[kb ^ 1], *S2 = slots[sbuf];
            pd_compact<<<grid(M, 256), 256, 0, st>>>(P, S, C, M, P2, S2);
            S = S2;
            sbuf ^= 1;
            M = kept;
            const int lo_bits = bitlen(N);
            bits = lo_bits + bitlen(N - 1);
            pd_key<<<grid(M, 256), 256, 0, st>>>(P2, rank, M, N, h, lo_bits, srt.k[kb ^ 1]);
            kb ^= 1;
            h *= 2;
        }
        if (!rc) {
            uint32_t r0 = 0;
            uint32_t *sa = reinterpret_cast<uint32_t *>(srt.k[0]);
            pd_sa<<<grid(N, 256), 256, 0, st>>>(rank, N, sa);
            if (cudaMemcpyAsync(&r0, rank, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                rc = GALN_ECUDA;
            primary = (uint64_t)r0 + 1;
            uint8_t *L = reinterpret_cast<uint8_t *>(srt.k[1]);
            U4 *cnt = reinterpret_cast<U4 *>(srt.v[0]);      // nb * 32 bytes <= 4N
            uint32_t *body = srt.v[1];                       // nb * 64 bytes <= 4N + 64
            uint64_t *smp = reinterpret_cast<uint64_t *>(slots[0]);
            if (!rc) {
                bwt_symbols<<<grid(N, 256), 256, 0, st>>>(T, sa, N, primary, L);
                bwt_block_counts<<<grid(nb, 128), 128, 0, st>>>(L, N, nb, cnt);
                rc = scan<U4, OpSum<U4>, true>(cnt, nb, scr, st);
            }
            if (!rc) {
                bwt_write<<<grid(nb * 16, 256), 256, 0, st>>>(L, N, nb, cnt, body);
                if (ns) sa_samples<<<grid(ns, 256), 256, 0, st>>>(sa, ns, smp);
                U4 totals{};
                cudaEventRecord(e1, st);
                cudaMemcpyAsync(bwt.data(), body, body_words * 4, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(&totals, cnt + nb - 1, sizeof(U4), cudaMemcpyDeviceToHost, st);
                if (ns) cudaMemcpyAsync(samples.data(), smp, ns * 8, cudaMemcpyDeviceToHost, st);
                cudaEventRecord(eb, st);
                if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = GALN_ECUDA;
                if (!rc) {
                    memcpy(bwt.data() + body_words, totals.c, sizeof(totals.c));
                    L2[0] = 0;
                    for (int c = 0; c < 4; ++c) L2[c + 1] = L2[c] + totals.c[c];
                }
            }
        }
        if (stats && !rc) {
            stats->n = N;
            stats->primary = primary;
            stats->rounds = rounds;
            stats->sorted_items = sorted;
            stats->sort_passes = srt.passes;
            stats->scatter_items = srt.scatter_items;
            float ms = 0, up = 0, down = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            cudaEventElapsedTime(&up, ea, e0);
            cudaEventElapsedTime(&down, e1, eb);
            stats->ms_device = ms;
            stats->ms_copies = up + down;
            double sc = 0;
            for (size_t i = 0; i + 1 < srt.ev.size(); i += 2) {
                float x = 0;
                cudaEventElapsedTime(&x, srt.ev[i], srt.ev[i + 1]);
                sc += x;
            }
            stats->ms_scatter = sc;
        }
        if (rc) cudaStreamSynchronize(st);
    }
    for (cudaEvent_t e : srt.ev) cudaEventDestroy(e);
    cudaEventDestroy(ea);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(eb);
    cudaStreamDestroy(st);
    if (rc == GALN_ECUDA) cudaGetLastError();
    return rc;
}

}  // namespace galn
