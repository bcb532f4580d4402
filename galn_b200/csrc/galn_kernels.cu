// galn_kernels.cu -- CUDA kernels of galn-b200 (sm_100a): index layout conversion, query encoding and the
// thread-per-read search tiers. Host-side orchestration is in galn_host.cpp.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "galn_internal.h"
#include "galn_search.cuh"
#include "galn_warp.cuh"

namespace galn {

static_assert(sizeof(HostBatchOpt) == sizeof(BatchOpt), "BatchOpt layout");

#define GALN_CUDA(call)                                                                          \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            fprintf(stderr, "[galn] CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            return -22;                                                                          \
        }                                                                                        \
    } while (0)

// ---------------------------------------------------------------------------------------------------
// bwa .bwt body -> occ64 blocks. Block b covers symbols [64b, 64b+64) of the $-free BWT; it sits in half
// (b & 1) of bwa block b >> 1 (128 symbols: 4 x uint64 counts, then 8 words of 16 symbols, first symbol
// in the top bits; src/index/idxcommon.c:72-112 writes that layout).
__global__ void convert_kernel(const uint32_t *__restrict__ body, uint64_t n_words, uint64_t n_sym,
                               uint64_t n_blocks, const uint64_t *__restrict__ sb, uint4 *__restrict__ out)
{
    uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_blocks) return;
    uint64_t B = b >> 1;
    int h = (int)(b & 1);
    const uint32_t *blk = body + B * 16;
    uint32_t words[4];
    for (int t = 0; t < 4; ++t) {
        uint64_t wi = B * 16 + 8 + 4 * h + t;
        uint64_t first_sym = 128 * B + 64 * h + 16 * t;
        words[t] = (wi < n_words && first_sym < n_sym) ? body[wi] : 0u;
    }
    uint64_t cnt[4] = {0, 0, 0, 0};
    if (B * 16 + 8 <= n_words) {
        for (int c = 0; c < 4; ++c) cnt[c] = (uint64_t)blk[2 * c] | ((uint64_t)blk[2 * c + 1] << 32);
    }
    if (h) {   // add the first 64 symbols of the bwa block
        for (int t = 0; t < 4; ++t) {
            uint64_t wi = B * 16 + 8 + t;
            uint32_t w = wi < n_words ? body[wi] : 0u;
            for (int j = 0; j < 16; ++j) {
                uint64_t sym_pos = 128 * B + 16 * t + j;
                if (sym_pos < n_sym) ++cnt[(w >> (30 - 2 * j)) & 3];
            }
        }
    }
    uint64_t p0 = 0, p1 = 0;
    for (int j = 0; j < 64; ++j) {
        uint64_t pos = 64 * b + j;
        if (pos >= n_sym) break;
        uint32_t s = (words[j >> 4] >> (30 - 2 * (j & 15))) & 3;
        p0 |= (uint64_t)(s & 1) << j;
        p1 |= (uint64_t)(s >> 1) << j;
    }
    const uint64_t *s = sb + ((64 * b) >> 32) * 4;
    out[2 * b] = make_uint4((uint32_t)(cnt[0] - s[0]), (uint32_t)(cnt[1] - s[1]), (uint32_t)(cnt[2] - s[2]),
                            (uint32_t)(cnt[3] - s[3]));
    out[2 * b + 1] = make_uint4((uint32_t)p0, (uint32_t)(p0 >> 32), (uint32_t)p1, (uint32_t)(p1 >> 32));
}

// occ64 blocks -> occ80 blocks. Block b covers symbols [80b, 80b+80): the counts of A, C, G before it
// (Occ at 80b - 1, relative to its superblock's sb80 entry) and the two bit planes of its 80 symbols, taken
// from the occ64 planes (positions past the text are 0 there and stay 0).
__global__ void convert80_kernel(const uint4 *__restrict__ occ64, uint64_t n_blocks64, const uint64_t *__restrict__ sb64,
                                 uint64_t n_blocks80, const uint64_t *__restrict__ sb80, uint4 *__restrict__ out)
{
    const uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_blocks80) return;
    const uint64_t start = 80 * b;
    uint64_t cnt[3] = {0, 0, 0};
    if (start > 0) {
        const uint64_t q = start - 1, B = q >> 6;
        const uint4 c = occ64[2 * B], x = occ64[2 * B + 1];
        const uint64_t p0 = (uint64_t)x.x | ((uint64_t)x.y << 32), p1 = (uint64_t)x.z | ((uint64_t)x.w << 32);
        const uint64_t m = (q & 63) == 63 ? ~0ull : (2ull << (q & 63)) - 1;
        const uint64_t *s = sb64 + (q >> 32) * 4;
        cnt[0] = s[0] + c.x + __popcll(~p0 & ~p1 & m);
        cnt[1] = s[1] + c.y + __popcll(p0 & ~p1 & m);
        cnt[2] = s[2] + c.z + __popcll(~p0 & p1 & m);
    }
    uint64_t w0[3], w1[3];   // planes 0 and 1 of occ64 blocks B0, B0+1, B0+2
    const uint64_t B0 = start >> 6;
    for (int t = 0; t < 3; ++t) {
        const uint64_t Bi = B0 + t;
        if (Bi < n_blocks64) {
            const uint4 x = occ64[2 * Bi + 1];
            w0[t] = (uint64_t)x.x | ((uint64_t)x.y << 32);
            w1[t] = (uint64_t)x.z | ((uint64_t)x.w << 32);
        } else w0[t] = w1[t] = 0;
    }
    const int off = (int)(start & 63);
    const uint64_t lo0 = off ? (w0[0] >> off) | (w0[1] << (64 - off)) : w0[0];
    const uint64_t lo1 = off ? (w1[0] >> off) | (w1[1] << (64 - off)) : w1[0];
    const uint64_t hi0 = off ? (w0[1] >> off) | (w0[2] << (64 - off)) : w0[1];
    const uint64_t hi1 = off ? (w1[1] >> off) | (w1[2] << (64 - off)) : w1[1];
    const uint64_t *base = sb80 + (b >> kOcc80SuperShift) * 4;
    out[2 * b] = make_uint4((uint32_t)(cnt[0] - base[0]), (uint32_t)(cnt[1] - base[1]), (uint32_t)(cnt[2] - base[2]),
                            (uint32_t)(hi0 & 0xffffu) | ((uint32_t)(hi1 & 0xffffu) << 16));
    out[2 * b + 1] = make_uint4((uint32_t)lo0, (uint32_t)(lo0 >> 32), (uint32_t)lo1, (uint32_t)(lo1 >> 32));
}

// Occ of each base before $-free position pos, from the .bwt body (per 128 symbols: 4 x u64 counts, then 8
// words of 16 symbols, first symbol in the top bits)
static void body_occ_before(const uint32_t *body, uint64_t n_words, uint64_t pos, uint64_t cnt[4])
{
    const uint64_t B = pos >> 7;
    for (int c = 0; c < 4; ++c) cnt[c] = (uint64_t)body[B * 16 + 2 * c] | ((uint64_t)body[B * 16 + 2 * c + 1] << 32);
    for (uint64_t p = B << 7; p < pos; ++p) {
        const uint64_t wi = B * 16 + 8 + ((p & 127) >> 4);
        const uint32_t w = wi < n_words ? body[wi] : 0u;
        ++cnt[(w >> (30 - 2 * (p & 15))) & 3];
    }
}

int dev_index_build(DevIndex &ix, const uint32_t *body, uint64_t n_words, cudaStream_t st)
{
    const uint64_t n = ix.seq_len;
    ix.n_blocks = n / 64 + 1;
    uint64_t n_super = (n >> 32) + 1;
    if (n_super > 16) return -20;
    // Occ before each superblock start (a multiple of 128: the stored counts of that bwa block)
    for (uint64_t s = 0; s < 16; ++s)
        for (int c = 0; c < 4; ++c) ix.sb[s][c] = 0;
    for (uint64_t s = 1; s < n_super; ++s) {
        uint64_t B = (s << 32) >> 7;
        for (int c = 0; c < 4; ++c) ix.sb[s][c] = (uint64_t)body[B * 16 + 2 * c] | ((uint64_t)body[B * 16 + 2 * c + 1] << 32);
    }
    GALN_CUDA(cudaSetDevice(ix.device));
    void *d_body = nullptr, *d_sb = nullptr;
    GALN_CUDA(cudaMalloc(&ix.blocks, ix.n_blocks * 32));
    GALN_CUDA(cudaMalloc(&d_body, n_words * 4));
    GALN_CUDA(cudaMalloc(&d_sb, sizeof(ix.sb)));
    GALN_CUDA(cudaMemcpyAsync(d_body, body, n_words * 4, cudaMemcpyHostToDevice, st));
    GALN_CUDA(cudaMemcpyAsync(d_sb, ix.sb, sizeof(ix.sb), cudaMemcpyHostToDevice, st));
    unsigned grid = (unsigned)((ix.n_blocks + 255) / 256);
    convert_kernel<<<grid, 256, 0, st>>>((const uint32_t *)d_body, n_words, n, ix.n_blocks, (const uint64_t *)d_sb,
                                         (uint4 *)ix.blocks);
    GALN_CUDA(cudaGetLastError());
    // the occ80 layout from the occ64 one
    ix.n_blocks80 = n / 80 + 1;
    const uint64_t n_super80 = (ix.n_blocks80 >> kOcc80SuperShift) + 1;
    if (n_super80 > 16) { cudaFree(d_body); cudaFree(d_sb); return -20; }
    for (uint64_t s = 0; s < 16; ++s)
        for (int c = 0; c < 4; ++c) ix.sb80[s][c] = 0;
    for (uint64_t s = 1; s < n_super80; ++s) body_occ_before(body, n_words, (s << kOcc80SuperShift) * 80, ix.sb80[s]);
    void *d_sb80 = nullptr;
    GALN_CUDA(cudaMalloc(&ix.blocks80, ix.n_blocks80 * 32));
    GALN_CUDA(cudaMalloc(&d_sb80, sizeof(ix.sb80)));
    GALN_CUDA(cudaMemcpyAsync(d_sb80, ix.sb80, sizeof(ix.sb80), cudaMemcpyHostToDevice, st));
    grid = (unsigned)((ix.n_blocks80 + 255) / 256);
    convert80_kernel<<<grid, 256, 0, st>>>((const uint4 *)ix.blocks, ix.n_blocks, (const uint64_t *)d_sb, ix.n_blocks80,
                                           (const uint64_t *)d_sb80, (uint4 *)ix.blocks80);
    GALN_CUDA(cudaGetLastError());
    GALN_CUDA(cudaStreamSynchronize(st));
    cudaFree(d_body);
    cudaFree(d_sb);
    cudaFree(d_sb80);
    return 0;
}

void dev_index_free(DevIndex &ix)
{
    cudaSetDevice(ix.device);
    if (ix.blocks) { cudaFree(ix.blocks); ix.blocks = nullptr; }
    if (ix.blocks80) { cudaFree(ix.blocks80); ix.blocks80 = nullptr; }
}

// ---------------------------------------------------------------------------------------------------
// query encoding: query[j] = complement(nt4(read[len-1-j])), ambiguous -> 4 (src/host_io.c:178-183)
__global__ void encode_kernel(const uint8_t *__restrict__ seq, const int64_t *__restrict__ off, int n,
                              uint8_t *__restrict__ query)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int64_t s = off[r], e = off[r + 1];
    int64_t len = e - s;
    for (int64_t j = 0; j < len; ++j) {
        uint8_t ch = seq[e - 1 - j];
        uint8_t b;
        switch (ch | 0x20) {
        case 'a': b = 3; break;    // complement of A
        case 'c': b = 2; break;
        case 'g': b = 1; break;
        case 't': b = 0; break;
        default: b = 4;
        }
        query[s + j] = b;
    }
}

int dev_encode(DevJob &job, cudaStream_t st)
{
    if (job.n_reads == 0) return 0;
    encode_kernel<<<(job.n_reads + 255) / 256, 256, 0, st>>>(job.seq, job.off, job.n_reads, job.query);
    GALN_CUDA(cudaGetLastError());
    return 0;
}

__device__ unsigned int g_l2_warm_sink;

// Reads every 16 bytes of p[0..n16) once through L2 (coalesced, not kept in L1), so that a search starting after
// other traffic finds the index in L2 instead of fetching it sector by sector at random.
__global__ void __launch_bounds__(256) l2_warm_kernel(const uint4 *p, size_t n16)
{
    uint32_t acc = 0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n16; t += (size_t)gridDim.x * blockDim.x) {
        const uint4 v = __ldcg(p + t);
        acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if (acc == 0x5bd1e995u && threadIdx.x == 0xffffu) g_l2_warm_sink = acc;   // keeps the loads; never true
}

int dev_l2_warm(const void *p, size_t bytes, int device, cudaStream_t st)
{
    if (!p || bytes < 16) return 0;
    int sms = 0;
    GALN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const size_t n16 = bytes / 16;
    const size_t want = (n16 + 255) / 256;
    const unsigned grid = (unsigned)std::min<size_t>(want, (size_t)std::max(sms, 1) * 8);
    l2_warm_kernel<<<grid, 256, 0, st>>>((const uint4 *)p, n16);
    GALN_CUDA(cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------------------------------
// search

struct KArgs {
    IndexView ix;
    const uint8_t *query;
    const int64_t *off;
    const int32_t *bidx;
    const int32_t *maxdiff;
    const BatchOpt *bopt;
    int seed_len;
    const int32_t *list;
    int n;
    int n_slots;            // workspace slots; threads at or past it do nothing
    int persistent;
    int32_t *claim;
    Workspace ws;
    int32_t *out_n;
    int64_t *out_off;
    uint64_t *out_pops, *out_trace;
    int32_t *out_peak;
    uint32_t *out_fetch;
    int8_t *out_tier;
    int tier;
    int trace;
    uint64_t *out_rec;
    unsigned long long *rec_top;
    int64_t rec_cap;
    int32_t *ovf;
    int32_t *ovf_n;
    // the fused launch: reads that overflow this tier and that the warp tier can take go to this queue
    // (hq_tail counts reserved slots) instead of ovf; NULL otherwise
    int32_t *hq;
    int32_t *hq_tail;
};

template <bool WIDE, bool FREELIST, bool TRACE, int S>
__device__ __forceinline__ void run_read(const KArgs &a, int pos, int slot)
{
    const int r = a.list[pos];
    const int64_t s = a.off[r];
    const int len = (int)(a.off[r + 1] - s);
    const uint8_t *q = a.query + s;
    const BatchOpt bo = a.bopt[a.bidx[r]];
    const int md = a.maxdiff[r];
    uint64_t *W = a.ws.wid + (size_t)slot * a.ws.wcap;
    uint64_t *SW = W + (len + 1);
    const bool use_seed = len > bo.seed_len;
    uint32_t fetches = 0;
    cal_width<S>(a.ix, len, q, W, fetches);
    if (use_seed) cal_width<S>(a.ix, bo.seed_len, q + (len - bo.seed_len), SW, fetches);
    SearchResult R = match_gap<WIDE, FREELIST, TRACE, S>(a.ix, bo, md, len, q, W, SW, use_seed, a.ws, slot, fetches);
    int ret = R.ret;
    if (ret > 0) {
        unsigned long long o = atomicAdd(a.rec_top, (unsigned long long)ret);
        if ((int64_t)(o + ret) > a.rec_cap) ret = kErrAln;
        else {
            const uint64_t *src = a.ws.aln + (size_t)slot * a.ws.aln_cap * 3;
            uint64_t *dst = a.out_rec + o * 3;
            for (int j = 0; j < 3 * ret; ++j) dst[j] = src[j];
            a.out_off[r] = (int64_t)o;
        }
    }
    a.out_n[r] = ret;
    a.out_pops[r] = R.pops;
    a.out_trace[r] = R.trace;
    a.out_peak[r] = R.peak;
    a.out_fetch[r] = R.fetches;
    a.out_tier[r] = (int8_t)a.tier;
    if (ret == kErrStack || ret == kErrAln) {
        // this tier's outputs are written before the read is handed on, so a warp that takes it from the
        // queue writes its own after them
        if (!WIDE && a.hq && len <= kWarpMaxLen && bo.n_stacks > 0 && bo.n_stacks <= kWarpMaxStacks && bo.s_mm > 0 &&
            bo.s_gapo > 0 && bo.s_gape > 0) {
            __threadfence();
            const int q = atomicAdd(a.hq_tail, 1);
            atomicExch(a.hq + q, r);
        } else a.ovf[atomicAdd(a.ovf_n, 1)] = r;
    }
}

template <bool WIDE, bool FREELIST, bool TRACE, int S>
__global__ void __launch_bounds__(512) search_kernel(const __grid_constant__ KArgs a)
{
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= a.n_slots) return;
    if (!a.persistent) {
        if (slot < a.n) run_read<WIDE, FREELIST, TRACE, S>(a, slot, slot);
        return;
    }
    for (;;) {
        int pos = atomicAdd(a.claim, 1);
        if (pos >= a.n) break;
        run_read<WIDE, FREELIST, TRACE, S>(a, pos, slot);
    }
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// width[] of the longest read, then seed_width[] when some read is longer than the seed
static int width_cap(const DevJob &job)
{
    return job.max_len + 1 + (job.max_len > job.seed_len ? job.seed_len + 1 : 0) + 1;
}

static void ws_layout(const TierCfg &cfg, const DevJob &job, size_t off[6])
{
    size_t slots = (size_t)cfg.threads;
    size_t esz = job.any_wide ? 32 : 16;
    int wcap = width_cap(job);
    off[0] = 0;
    off[1] = off[0] + align256(slots * cfg.cap * esz);
    off[2] = off[1] + align256(slots * cfg.cap * 4);
    off[3] = off[2] + align256(slots * (size_t)job.max_stacks * 4);
    off[4] = off[3] + align256(slots * (size_t)wcap * 8);
    off[5] = off[4] + align256(slots * (size_t)cfg.aln_cap * 24);
}

size_t ws_bytes(const TierCfg &cfg, const DevJob &job)
{
    size_t off[6];
    ws_layout(cfg, job, off);
    return off[5];
}

template <bool WIDE, bool FREELIST, int S>
static int launch(const KArgs &a, int threads, int block, cudaStream_t st)
{
    unsigned grid = (unsigned)((threads + block - 1) / block);
    if (a.trace) search_kernel<WIDE, FREELIST, true, S><<<grid, block, 0, st>>>(a);
    else search_kernel<WIDE, FREELIST, false, S><<<grid, block, 0, st>>>(a);
    GALN_CUDA(cudaGetLastError());
    return 0;
}

template <int S>
static int launch_s(const KArgs &a, bool wide, bool freelist, int threads, int block, cudaStream_t st)
{
    if (wide) return freelist ? launch<true, true, S>(a, threads, block, st) : launch<true, false, S>(a, threads, block, st);
    return freelist ? launch<false, true, S>(a, threads, block, st) : launch<false, false, S>(a, threads, block, st);
}

// the kernels' view of the index in the job's occurrence layout
static int index_view(const DevIndex &ix, int occ, IndexView &v)
{
    if (occ != kOcc64 && occ != kOcc80) return -20;
    if (occ == kOcc80 && !ix.blocks80) return -20;
    v.blk = (const uint4 *)(occ == kOcc64 ? ix.blocks : ix.blocks80);
    v.primary = ix.primary;
    v.seq_len = ix.seq_len;
    for (int c = 0; c < 4; ++c) v.C[c] = ix.L2[c];
    memcpy(v.sb, occ == kOcc64 ? ix.sb : ix.sb80, sizeof(v.sb));
    return 0;
}

int dev_search(const DevIndex &ix, DevJob &job, const TierCfg &cfg, const int32_t *list, int n, int32_t *ovf,
               void *ws_mem, cudaStream_t st)
{
    if (n == 0) return 0;
    KArgs a;
    memset(&a, 0, sizeof(a));
    if (index_view(ix, job.occ, a.ix)) return -20;
    a.query = job.query; a.off = job.off; a.bidx = job.bidx; a.maxdiff = job.maxdiff;
    a.bopt = (const BatchOpt *)job.bopt; a.seed_len = job.seed_len;
    a.list = list; a.n = n; a.persistent = cfg.persistent ? 1 : 0; a.claim = job.counters;
    a.n_slots = cfg.threads;
    size_t off[6];
    ws_layout(cfg, job, off);
    char *base = (char *)ws_mem;
    a.ws.ent = (uint4 *)(base + off[0]);
    a.ws.link = (int32_t *)(base + off[1]);
    a.ws.heads = (int32_t *)(base + off[2]);
    a.ws.wid = (uint64_t *)(base + off[3]);
    a.ws.aln = (uint64_t *)(base + off[4]);
    a.ws.cap = cfg.cap; a.ws.hcap = job.max_stacks; a.ws.wcap = width_cap(job);
    a.ws.aln_cap = cfg.aln_cap;
    a.out_n = job.out_n; a.out_off = job.out_off; a.out_pops = job.out_pops; a.out_trace = job.out_trace;
    a.out_peak = job.out_peak; a.out_fetch = job.out_fetch; a.out_tier = job.out_tier; a.tier = cfg.tier;
    a.trace = job.trace;
    a.out_rec = job.out_rec; a.rec_top = job.rec_top; a.rec_cap = job.rec_cap;
    a.ovf = ovf; a.ovf_n = job.counters + 1;
    if (!cfg.persistent && cfg.threads < n) return -20;
    int threads = cfg.persistent ? cfg.threads : n;
    if (job.occ == kOcc80) return launch_s<kOcc80>(a, job.any_wide, cfg.freelist, threads, cfg.block, st);
    return launch_s<kOcc64>(a, job.any_wide, cfg.freelist, threads, cfg.block, st);
}

int dev_resident_threads(const TierCfg &cfg, bool wide, int device)
{
    int bps = 0;
    cudaError_t e;
    // the smallest residency over the layouts and trace modes of this tier's kernel
    const void *fns[4];
    if (wide && cfg.freelist) {
        fns[0] = (const void *)search_kernel<true, true, true, kOcc64>; fns[1] = (const void *)search_kernel<true, true, false, kOcc64>;
        fns[2] = (const void *)search_kernel<true, true, true, kOcc80>; fns[3] = (const void *)search_kernel<true, true, false, kOcc80>;
    } else if (wide) {
        fns[0] = (const void *)search_kernel<true, false, true, kOcc64>; fns[1] = (const void *)search_kernel<true, false, false, kOcc64>;
        fns[2] = (const void *)search_kernel<true, false, true, kOcc80>; fns[3] = (const void *)search_kernel<true, false, false, kOcc80>;
    } else if (cfg.freelist) {
        fns[0] = (const void *)search_kernel<false, true, true, kOcc64>; fns[1] = (const void *)search_kernel<false, true, false, kOcc64>;
        fns[2] = (const void *)search_kernel<false, true, true, kOcc80>; fns[3] = (const void *)search_kernel<false, true, false, kOcc80>;
    } else {
        fns[0] = (const void *)search_kernel<false, false, true, kOcc64>; fns[1] = (const void *)search_kernel<false, false, false, kOcc64>;
        fns[2] = (const void *)search_kernel<false, false, true, kOcc80>; fns[3] = (const void *)search_kernel<false, false, false, kOcc80>;
    }
    e = cudaSuccess;
    bps = 1 << 30;
    for (const void *f : fns) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, cfg.block, 0) != cudaSuccess) { e = cudaErrorInvalidValue; break; }
        bps = std::min(bps, b);
    }
    if (e != cudaSuccess) return -22;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return bps * cfg.block * sms;
}

// ---------------------------------------------------------------------------------------------------
// the warp tier

size_t warp_smem_bytes() { return sizeof(WarpSmem); }

int warp_resident(int device)
{
    int bps = 0;
    size_t smem = sizeof(WarpSmem);
    const void *fns[4] = {(const void *)warp_kernel<false, kOcc64>, (const void *)warp_kernel<true, kOcc64>,
                          (const void *)warp_kernel<false, kOcc80>, (const void *)warp_kernel<true, kOcc80>};
    bps = 1 << 30;
    for (const void *f : fns) {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, 32, smem) != cudaSuccess) return -22;
        bps = std::min(bps, b);
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return bps * sms;
}

// ---- suffix-array positions (the coordinate step of samse: bwt_sa, bwa_sa2pos) ----
// bwt_sa (bwa's bwt.c:86-96, as used by samse/bwa_upstream/bwase.c:112-125): from row k, step back with
// invPsi(k) = L2[c] + Occ(c, k) (c = the row's BWT symbol; the $ row goes to 0) until k is a multiple of the
// sampling interval, then add the steps to the sample (sample 0, the $ row, is -1). One thread per query;
// each step reads one occ64 block, which holds both the symbol and its count.
__global__ void sa_walk_kernel(IndexView ix, const uint64_t *__restrict__ samples, uint64_t intv_mask, int intv_shift,
                               const uint64_t *__restrict__ k_in, int64_t n, const int32_t *__restrict__ ref_len,
                               uint64_t l_pac, uint64_t *__restrict__ pos_out, int8_t *__restrict__ strand_out)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    uint64_t k = k_in[t], sa = 0;
    if (k > ix.seq_len) { pos_out[t] = ~0ull; if (strand_out) strand_out[t] = 0; return; }
    while (k & intv_mask) {
        ++sa;
        if (k == ix.primary) { k = 0; continue; }
        const uint64_t p = k - (k >= ix.primary);         // the row's $-free position
        const uint4 *b = ix.blk + ((p >> 6) << 1);
        const uint4 cnt = __ldg(b), bits = __ldg(b + 1);
        const uint64_t p0 = (uint64_t)bits.x | ((uint64_t)bits.y << 32), p1 = (uint64_t)bits.z | ((uint64_t)bits.w << 32);
        const int j = (int)(p & 63);
        const int c = (int)(((p0 >> j) & 1) | (((p1 >> j) & 1) << 1));
        const uint64_t m = j == 63 ? ~0ull : (2ull << j) - 1;
        const uint64_t a = c & 1 ? p0 : ~p0, h = c & 2 ? p1 : ~p1;
        const uint32_t cc = c == 0 ? cnt.x : c == 1 ? cnt.y : c == 2 ? cnt.z : cnt.w;
        k = ix.C[c] + ix.sb[p >> 32][c] + cc + __popcll(a & h & m);
    }
    uint64_t pos_f = sa + samples[k >> intv_shift];
    if (!ref_len) { pos_out[t] = pos_f; return; }
    // bwa_sa2pos: a hit across the forward/reverse boundary has no position; on the reverse half the
    // position is mirrored and moved to the hit's first base
    const uint64_t rl = (uint64_t)(int64_t)ref_len[t];
    if (pos_f < l_pac && l_pac < pos_f + rl) { pos_out[t] = ~0ull; strand_out[t] = 0; return; }
    const bool rev = pos_f >= l_pac;
    if (rev) pos_f = (l_pac << 1) - 1 - pos_f;
    if (rev) pos_f = pos_f + 1 < rl ? 0 : pos_f - rl + 1;
    pos_out[t] = pos_f;
    strand_out[t] = rev ? 0 : 1;
}

int dev_sa_walk(const DevIndex &ix, const uint64_t *d_samples, uint64_t intv, const uint64_t *d_k, int64_t n,
                const int32_t *d_ref_len, uint64_t *d_pos, int8_t *d_strand, cudaStream_t st)
{
    if (n <= 0) return 0;
    if (intv == 0 || (intv & (intv - 1))) return -20;
    IndexView v;
    if (index_view(ix, kOcc64, v)) return -20;
    int shift = 0;
    while ((1ull << shift) < intv) ++shift;
    const unsigned grid = (unsigned)((n + 255) / 256);
    sa_walk_kernel<<<grid, 256, 0, st>>>(v, d_samples, intv - 1, shift, d_k, n, d_ref_len, ix.seq_len / 2, d_pos, d_strand);
    GALN_CUDA(cudaGetLastError());
    return 0;
}

// ---- the occurrence layer on its own: Occ of the four bases at BWT rows, for checks ----
template <int S>
__global__ void occ_probe_kernel(IndexView ix, const uint64_t *__restrict__ rows, int64_t n, uint64_t *__restrict__ occ,
                                 uint32_t *__restrict__ fetch)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    uint64_t ok[4], ol[4];
    uint32_t f = 0;
    occ4_pair_u<S>(ix, rows[t], rows[t], ok, ol, f);
#pragma unroll
    for (int c = 0; c < 4; ++c) occ[4 * t + c] = ok[c];
    if (fetch) fetch[t] = f;
}

int dev_occ_probe(const DevIndex &ix, int occ, const uint64_t *d_rows, int64_t n, uint64_t *d_occ, uint32_t *d_fetch,
                  cudaStream_t st)
{
    if (n <= 0) return 0;
    IndexView v;
    if (index_view(ix, occ, v)) return -20;
    const unsigned grid = (unsigned)((n + 255) / 256);
    if (occ == kOcc80) occ_probe_kernel<kOcc80><<<grid, 256, 0, st>>>(v, d_rows, n, d_occ, d_fetch);
    else occ_probe_kernel<kOcc64><<<grid, 256, 0, st>>>(v, d_rows, n, d_occ, d_fetch);
    GALN_CUDA(cudaGetLastError());
    return 0;
}

// ---- random 32-byte gather peak (a measurement, not part of the search) ----
// Every thread reads `per_thread` 32-byte sectors at pseudo-random sector indices of a power-of-two buffer
// (a splitmix64 sequence per thread; IF independent sectors in flight per thread, each read as the search
// reads an index block: two 16-byte loads), and folds them into one word so the loads are not dead. Bytes
// read / time is the device's random-sector read rate for that buffer size and depth of loads in flight.
__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

template <int IF>
__global__ void __launch_bounds__(256) gather_kernel(const uint4 *buf, uint64_t sector_mask, int per_thread, uint32_t *sink)
{
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = 0;
    for (int i = 0; i < per_thread; i += IF) {
        uint4 a[IF], b[IF];
#pragma unroll
        for (int u = 0; u < IF; ++u) {
            const uint64_t sct = mix64(tid * 0x100000001b3ull + (uint64_t)(i + u)) & sector_mask;
            a[u] = __ldcg(buf + 2 * sct);
            b[u] = __ldcg(buf + 2 * sct + 1);
        }
#pragma unroll
        for (int u = 0; u < IF; ++u) acc ^= a[u].x ^ a[u].w ^ b[u].y ^ b[u].z;
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;   // practically never; keeps the loads
}

extern "C" int galn_gather_peak_ex(int device, uint64_t bytes, int in_flight, int repeats, double *gbs)
{
    if (!gbs || bytes < (1u << 20) || repeats < 1) return -20;
    if (in_flight != 2 && in_flight != 4 && in_flight != 8 && in_flight != 16) return -20;
    while (bytes & (bytes - 1)) bytes &= bytes - 1;      // the largest power of two not above it
    if (cudaSetDevice(device) != cudaSuccess) return -22;
    void *buf = nullptr, *sink = nullptr;
    if (cudaMalloc(&buf, bytes) != cudaSuccess) { cudaGetLastError(); return -23; }
    if (cudaMalloc(&sink, 64) != cudaSuccess) { cudaFree(buf); cudaGetLastError(); return -23; }
    cudaMemset(buf, 0x5a, bytes);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, per_thread = 256;
    const uint64_t sector_mask = bytes / 32 - 1;
    auto launch = [&]() {
        const uint4 *b = (const uint4 *)buf;
        uint32_t *k = (uint32_t *)sink;
        switch (in_flight) {
        case 2: gather_kernel<2><<<blocks, 256>>>(b, sector_mask, per_thread, k); break;
        case 4: gather_kernel<4><<<blocks, 256>>>(b, sector_mask, per_thread, k); break;
        case 8: gather_kernel<8><<<blocks, 256>>>(b, sector_mask, per_thread, k); break;
        default: gather_kernel<16><<<blocks, 256>>>(b, sector_mask, per_thread, k); break;
        }
    };
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch();   // warm-up
    double best = 0;
    for (int r = 0; r < repeats; ++r) {
        cudaEventRecord(e0);
        launch();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double v = (double)blocks * 256 * per_thread * 32 / (ms * 1e-3) / 1e9;
        if (v > best) best = v;
    }
    const cudaError_t ce = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    cudaFree(sink);
    if (ce != cudaSuccess) return -22;
    *gbs = best;
    return 0;
}

extern "C" int galn_gather_peak(int device, uint64_t bytes, int repeats, double *gbs)
{
    return galn_gather_peak_ex(device, bytes, 8, repeats, gbs);
}

// ---- results in read order ----
// Records are appended to out_rec in the order reads finish (an atomic counter per record block); the caller
// wants them in read order. An exclusive scan of max(n_aln, 0) gives each read's first record in read order;
// the last kernel adds the block prefixes and gathers each read's records there.
constexpr int kScanThreads = 1024, kScanItems = 4, kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t *sm, int64_t &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sm[w] = x;
    __syncthreads();
    if (w == 0) {
        int64_t s = lane < kScanThreads / 32 ? sm[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        sm[lane] = s;     // inclusive prefix of warp sums
    }
    __syncthreads();
    total = sm[kScanThreads / 32 - 1];
    const int64_t before = w ? sm[w - 1] : 0;
    __syncthreads();
    return before + x - v;
}

// per tile: local exclusive offsets into rec_off[], tile sums into tile_sum[]
__global__ void __launch_bounds__(kScanThreads) scan_tiles_kernel(const int32_t *n_aln, int n, int64_t *rec_off,
                                                                  int64_t *tile_sum)
{
    __shared__ int64_t sm[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems], s = 0;
#pragma unroll
    for (int u = 0; u < kScanItems; ++u) {
        const int64_t r = base + u;
        v[u] = r < n ? (int64_t)max(n_aln[r], 0) : 0;
        s += v[u];
    }
    int64_t total;
    int64_t off = block_excl_scan(s, sm, total);
#pragma unroll
    for (int u = 0; u < kScanItems; ++u) {
        const int64_t r = base + u;
        if (r < n) rec_off[r] = off;
        off += v[u];
    }
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// exclusive scan of the tile sums, in one block; the grand total goes to rec_off[n]
__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(int64_t *tile_sum, int n_tiles, int64_t *rec_off, int n)
{
    __shared__ int64_t sm[32];
    int64_t carry = 0;
    for (int t0 = 0; t0 < n_tiles; t0 += kScanThreads) {
        const int t = t0 + threadIdx.x;
        const int64_t v = t < n_tiles ? tile_sum[t] : 0;
        int64_t total;
        const int64_t e = block_excl_scan(v, sm, total);
        if (t < n_tiles) tile_sum[t] = carry + e;
        carry += total;
    }
    if (threadIdx.x == 0) rec_off[n] = carry;
}

// add the tile prefix; copy each read's records (3 words each) to their place in read order
__global__ void __launch_bounds__(kScanThreads) gather_records_kernel(const int32_t *n_aln, const int64_t *dev_off,
                                                                      const uint64_t *rec, int n, int64_t *rec_off,
                                                                      const int64_t *tile_sum, uint64_t *rec_ord)
{
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    const int64_t add = tile_sum[blockIdx.x];
#pragma unroll
    for (int u = 0; u < kScanItems; ++u) {
        const int64_t r = base + u;
        if (r >= n) break;
        const int64_t o = rec_off[r] + add;
        rec_off[r] = o;
        const int k = n_aln[r];
        for (int j = 0; j < 3 * k; ++j) rec_ord[3 * o + j] = rec[3 * dev_off[r] + j];
    }
}

int dev_order_results(const DevJob &job, int n, int64_t *rec_off, uint64_t *rec_ord, int64_t *tile_sum, cudaStream_t st)
{
    if (n <= 0) return 0;
    const int tiles = (int)(((int64_t)n + kScanTile - 1) / kScanTile);
    scan_tiles_kernel<<<tiles, kScanThreads, 0, st>>>(job.out_n, n, rec_off, tile_sum);
    scan_sums_kernel<<<1, kScanThreads, 0, st>>>(tile_sum, tiles, rec_off, n);
    gather_records_kernel<<<tiles, kScanThreads, 0, st>>>(job.out_n, job.out_off, job.out_rec, n, rec_off, tile_sum, rec_ord);
    GALN_CUDA(cudaGetLastError());
    return 0;
}

size_t order_tile_bytes(int n) { return ((size_t)std::max(n, 1) + kScanTile - 1) / kScanTile * 8 + 8; }

// workspace layout of the warp tier, in order
struct WarpLayout {
    size_t chunks, chunk_prev, free_ids, aln, stage, prec, side, q_ctl, ovq, total;
};

static WarpLayout warp_layout(const WarpCfg &c, int n)
{
    const size_t w = (size_t)c.n_warps;
    const size_t tot = (size_t)c.n_big * c.big_chunks + (w - (size_t)c.n_big) * c.arena_chunks;
    WarpLayout L;
    size_t o = 0;
    L.chunks = o;     o += align256(tot * kWCH * 16);
    L.chunk_prev = o; o += align256(tot * 4);
    L.free_ids = o;   o += align256(tot * 4);
    L.aln = o;        o += align256(w * c.aln_cap * 24);
    L.stage = o;      o += align256(w * 3 * 32 * kWL * 16);
    L.prec = o;       o += align256(w * 32 * kWP * 16);
    L.side = o;       o += align256(w * sizeof(WSide));
    L.q_ctl = o;      o += align256(16);
    L.ovq = o;        o += align256((size_t)std::max(n, 1) * 4);
    L.total = o;
    return L;
}

size_t warp_ws_bytes(const WarpCfg &c, int n) { return warp_layout(c, n).total; }

int32_t *warp_queue(const WarpCfg &c, int n, void *ws_mem, int32_t **slots)
{
    const WarpLayout L = warp_layout(c, n);
    *slots = (int32_t *)((char *)ws_mem + L.ovq);
    return (int32_t *)((char *)ws_mem + L.q_ctl);
}

int dev_search_warp(const DevIndex &ix, DevJob &job, const WarpCfg &c, int tier, const int32_t *list, int n,
                    int32_t *ovf, void *ws_mem, cudaStream_t st, unsigned long long *dbg)
{
    if (n == 0) return 0;
    if (c.n_big < 0 || c.n_big > c.n_warps || (c.n_big > 0 && c.big_chunks < 1) || c.arena_chunks < 1) return -20;   // GALN_EINVAL
    WArgs a;
    memset(&a, 0, sizeof(a));
    if (index_view(ix, job.occ, a.ix)) return -20;
    a.query = job.query; a.off = job.off; a.bidx = job.bidx; a.maxdiff = job.maxdiff;
    a.bopt = (const BatchOpt *)job.bopt; a.seed_len = job.seed_len;
    a.list = list; a.n = n; a.claim = job.counters; a.n_warps = c.n_warps;
    const WarpLayout L = warp_layout(c, n);
    char *base = (char *)ws_mem;
    a.chunks = (uint4 *)(base + L.chunks);
    a.chunk_prev = (int32_t *)(base + L.chunk_prev);
    a.free_ids = (int32_t *)(base + L.free_ids);
    a.aln = (uint64_t *)(base + L.aln);
    a.stage = (uint4 *)(base + L.stage);
    a.prec = (uint4 *)(base + L.prec);
    a.side = (WSide *)(base + L.side);
    a.q_ctl = (int32_t *)(base + L.q_ctl);
    a.ovq = (int32_t *)(base + L.ovq);
    a.n_big = c.n_big; a.big_chunks = c.big_chunks; a.q_wait_ns = c.q_wait_ns;
    GALN_CUDA(cudaMemsetAsync(a.q_ctl, 0, 16, st));
    GALN_CUDA(cudaMemsetAsync(a.ovq, 0xff, (size_t)n * 4, st));
    const int arena_chunks = c.arena_chunks, aln_cap = c.aln_cap, n_warps = c.n_warps;
    a.arena_chunks = arena_chunks; a.aln_cap = aln_cap;
    a.out_n = job.out_n; a.out_off = job.out_off; a.out_pops = job.out_pops; a.out_trace = job.out_trace;
    a.out_peak = job.out_peak; a.out_fetch = job.out_fetch; a.out_tier = job.out_tier; a.tier = tier;
    a.out_rec = job.out_rec; a.rec_top = job.rec_top; a.rec_cap = job.rec_cap;
    a.ovf = ovf; a.ovf_n = job.counters + 1;
    a.dbg = dbg;
    size_t smem = sizeof(WarpSmem);
    if (job.occ == kOcc80) {
        if (job.trace) warp_kernel<true, kOcc80><<<n_warps, 32, smem, st>>>(a);
        else warp_kernel<false, kOcc80><<<n_warps, 32, smem, st>>>(a);
    } else {
        if (job.trace) warp_kernel<true, kOcc64><<<n_warps, 32, smem, st>>>(a);
        else warp_kernel<false, kOcc64><<<n_warps, 32, smem, st>>>(a);
    }
    GALN_CUDA(cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------------------------------
// The fused launch: the first tier and the warp tier in one persistent launch. Blocks of kFWarps warps; the
// first n_w_blocks blocks are warp-tier warps from the start, the others run the first tier (one read per
// thread, claimed from the list) and then become warp-tier warps too. A read that overflows the first tier
// and that the warp tier can take is handed over at once through the heavy queue (hq), so heavy reads start
// while light ones are still being searched. Every wait is bounded (w.q_wait_ns): a warp that gives up
// leaves its reads to the host's next pass, and a lost queue slot is flagged (hq_ctl[3]) so that the host
// searches every queued read again; results never depend on any of it.
constexpr int kFWarps = kFusedWarps;

struct FArgs {
    KArgs t;                 // the first tier; t.hq / t.hq_tail point into hq / hq_ctl
    WArgs w;                 // the warp tier (w.list, w.n and w.claim are unused: reads come from hq)
    int n_w_blocks;          // blocks that are warp-tier warps from the start (they come first)
    int32_t *hq;             // heavy queue: read ids, -1 until written
    int32_t *hq_ctl;         // 0 head (claimed), 1 tail (reserved), 2 first-tier warps still running, 3 a slot was lost
};

// takes slot `h` of a queue whose producers reserve a slot and then write the read id into it
__device__ __forceinline__ int queue_take(int32_t *q, int h, uint64_t t0, uint64_t wait, int32_t *lost)
{
    for (;;) {
        const int r = atomicAdd(q + h, 0);
        if (r >= 0) { __threadfence(); return r; }
        if (gtimer_ns() - t0 > wait) { atomicExch(lost, 1); return -1; }
        __nanosleep(100);
    }
}

// a small warp's next read (lane 0): the next heavy read; -1 once the first tier has finished and the queue
// is empty, or when the first tier has shown no progress (reads claimed, reads queued, warps finished) for
// w.q_wait_ns
__device__ __noinline__ int heavy_next(const FArgs &f)
{
    volatile int32_t *hc = f.hq_ctl;
    volatile int32_t *claim = f.t.claim;
    uint64_t t0 = gtimer_ns();
    int seen_t = hc[1], seen_w = hc[2], seen_c = *claim;
    for (;;) {
        const int h = hc[0], t = hc[1];
        if (h < t) {
            if (atomicCAS(f.hq_ctl, h, h + 1) == h) return queue_take(f.hq, h, gtimer_ns(), f.w.q_wait_ns, f.hq_ctl + 3);
            continue;
        }
        const int w = hc[2], c = *claim;
        if (w == 0) {
            __threadfence();
            if (hc[0] >= hc[1]) return -1;
            continue;
        }
        const uint64_t now = gtimer_ns();
        if (t != seen_t || w != seen_w || c != seen_c) { seen_t = t; seen_w = w; seen_c = c; t0 = now; }
        else if (now - t0 > f.w.q_wait_ns) {               // reads queued later go to the host's next pass
            if (f.w.q_wait_ns == 0) atomicExch(f.hq_ctl + 3, 1);
            return -1;
        }
        __nanosleep(1000);
    }
}

// a big warp's next read (lane 0): one that outgrew a small arena first, else a heavy read; -1 once every
// small warp has finished and both queues are empty, or after a wait of w.q_wait_ns
__device__ __noinline__ int fused_big_next(const FArgs &f)
{
    volatile int32_t *qc = f.w.q_ctl;
    volatile int32_t *hc = f.hq_ctl;
    const int n_small = f.w.n_warps - f.w.n_big;
    const uint64_t t0 = gtimer_ns();
    for (;;) {
        const int h = qc[0], t = qc[1];
        if (h < t) {
            if (atomicCAS(f.w.q_ctl, h, h + 1) == h)
                return queue_take(f.w.ovq, h, gtimer_ns(), f.w.q_wait_ns, f.w.q_ctl + 3);
            continue;
        }
        const int h2 = hc[0], t2 = hc[1];
        if (h2 < t2) {
            if (atomicCAS(f.hq_ctl, h2, h2 + 1) == h2)
                return queue_take(f.hq, h2, gtimer_ns(), f.w.q_wait_ns, f.hq_ctl + 3);
            continue;
        }
        if (qc[2] == n_small) {
            __threadfence();
            if (qc[0] >= qc[1]) return -1;
            continue;
        }
        if (gtimer_ns() - t0 > f.w.q_wait_ns) {
            if (f.w.q_wait_ns == 0) atomicExch(f.w.q_ctl + 3, 1);
            return -1;
        }
        __nanosleep(1000);
    }
}

template <bool TRACE, int ST>
__global__ void __launch_bounds__(kFWarps * 32, 2) fused_kernel(const __grid_constant__ FArgs f)
{
    extern __shared__ __align__(16) unsigned char fsm_raw[];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpSmem *S = reinterpret_cast<WarpSmem *>(fsm_raw) + wib;
    const int wid = blockIdx.x * kFWarps + wib;
    if ((int)blockIdx.x >= f.n_w_blocks) {
        const int slot = ((int)blockIdx.x - f.n_w_blocks) * kFWarps * 32 + threadIdx.x;
        if (slot < f.t.n_slots) {
            for (;;) {
                const int pos = atomicAdd(f.t.claim, 1);
                if (pos >= f.t.n) break;
                run_read<false, false, TRACE, ST>(f.t, pos, slot);
            }
        }
        __syncwarp();
        if (lane == 0) {
            __threadfence();
            atomicSub(f.hq_ctl + 2, 1);
        }
    }
    const bool big = wid < f.w.n_big;
    for (;;) {
        int r = -1;
        if (lane == 0) r = big ? fused_big_next(f) : heavy_next(f);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r < 0) break;
        warp_read<TRACE, ST>(f.w, r, wid, S, lane);
    }
    if (!big && f.w.n_big > 0 && lane == 0) {
        __threadfence();
        atomicAdd(f.w.q_ctl + 2, 1);
    }
}

__global__ void fused_init_kernel(int32_t *hq_ctl, int32_t *q_ctl, int t0_warps)
{
    if (threadIdx.x < 4) {
        hq_ctl[threadIdx.x] = threadIdx.x == 2 ? t0_warps : 0;
        q_ctl[threadIdx.x] = 0;
    }
}

size_t fused_smem_bytes() { return (size_t)kFWarps * sizeof(WarpSmem); }

// blocks of the fused kernel resident per SM (its registers and shared memory allow)
int fused_resident_blocks(int device)
{
    const void *fns[4] = {(const void *)fused_kernel<false, kOcc64>, (const void *)fused_kernel<true, kOcc64>,
                          (const void *)fused_kernel<false, kOcc80>, (const void *)fused_kernel<true, kOcc80>};
    int bps = 1 << 30;
    for (const void *fn : fns) {
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_smem_bytes()) != cudaSuccess)
            return -22;
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kFWarps * 32, fused_smem_bytes()) != cudaSuccess)
            return -22;
        bps = std::min(bps, b);
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return bps * sms;
}

// workspace: the first tier's (t0.threads slots), the warp tier's (c.n_warps warps), the heavy queue (n slots)
// and its control words, and the warp tier's overflow list (n slots)
struct FusedLayout {
    size_t t0, warp, hq, hq_ctl, w_ovf, total;
};

static FusedLayout fused_layout(const TierCfg &t0, const DevJob &job, const WarpCfg &c, int n)
{
    FusedLayout L;
    size_t o = 0;
    L.t0 = o;     o += align256(ws_bytes(t0, job));
    L.warp = o;   o += align256(warp_ws_bytes(c, n));
    L.hq = o;     o += align256((size_t)std::max(n, 1) * 4);
    L.hq_ctl = o; o += 256;
    L.w_ovf = o;  o += align256((size_t)std::max(n, 1) * 4);
    L.total = o;
    return L;
}

size_t fused_ws_bytes(const TierCfg &t0, const DevJob &job, const WarpCfg &c, int n)
{
    return fused_layout(t0, job, c, n).total;
}

void fused_queues(const TierCfg &t0, const DevJob &job, const WarpCfg &c, int n, void *ws_mem, FusedQueues &q)
{
    const FusedLayout L = fused_layout(t0, job, c, n);
    char *b = (char *)ws_mem;
    q.hq = (int32_t *)(b + L.hq);
    q.hq_ctl = (int32_t *)(b + L.hq_ctl);
    q.w_ovf = (int32_t *)(b + L.w_ovf);
    q.q_ctl = warp_queue(c, n, b + L.warp, &q.big_slots);
}

int dev_search_fused(const DevIndex &ix, DevJob &job, const TierCfg &t0, const WarpCfg &c, int n_w_blocks,
                     const int32_t *list, int n, int32_t *t0_ovf, void *ws_mem, cudaStream_t st, unsigned long long *dbg)
{
    if (n == 0) return 0;
    const int grid = c.n_warps / kFWarps;
    if (c.n_warps % kFWarps || grid <= n_w_blocks || n_w_blocks < 0 || t0.threads != (grid - n_w_blocks) * kFWarps * 32 ||
        c.n_big < 0 || c.n_big > n_w_blocks * kFWarps || (c.n_big > 0 && c.big_chunks < 1) || c.arena_chunks < 1 ||
        job.any_wide)
        return -20;
    const FusedLayout L = fused_layout(t0, job, c, n);
    char *base = (char *)ws_mem;
    FArgs f;
    memset(&f, 0, sizeof(f));
    // the first tier
    KArgs &a = f.t;
    if (index_view(ix, job.occ, a.ix)) return -20;
    a.query = job.query; a.off = job.off; a.bidx = job.bidx; a.maxdiff = job.maxdiff;
    a.bopt = (const BatchOpt *)job.bopt; a.seed_len = job.seed_len;
    a.list = list; a.n = n; a.persistent = 1; a.claim = job.counters;
    a.n_slots = t0.threads;
    size_t off[6];
    ws_layout(t0, job, off);
    char *tb = base + L.t0;
    a.ws.ent = (uint4 *)(tb + off[0]);
    a.ws.link = (int32_t *)(tb + off[1]);
    a.ws.heads = (int32_t *)(tb + off[2]);
    a.ws.wid = (uint64_t *)(tb + off[3]);
    a.ws.aln = (uint64_t *)(tb + off[4]);
    a.ws.cap = t0.cap; a.ws.hcap = job.max_stacks; a.ws.wcap = width_cap(job);
    a.ws.aln_cap = t0.aln_cap;
    a.out_n = job.out_n; a.out_off = job.out_off; a.out_pops = job.out_pops; a.out_trace = job.out_trace;
    a.out_peak = job.out_peak; a.out_fetch = job.out_fetch; a.out_tier = job.out_tier; a.tier = 0;
    a.trace = job.trace;
    a.out_rec = job.out_rec; a.rec_top = job.rec_top; a.rec_cap = job.rec_cap;
    a.ovf = t0_ovf; a.ovf_n = job.counters + 1;
    f.hq = (int32_t *)(base + L.hq);
    f.hq_ctl = (int32_t *)(base + L.hq_ctl);
    a.hq = f.hq; a.hq_tail = f.hq_ctl + 1;
    // the warp tier
    WArgs &w = f.w;
    w.ix = a.ix;
    w.query = job.query; w.off = job.off; w.bidx = job.bidx; w.maxdiff = job.maxdiff;
    w.bopt = a.bopt; w.seed_len = job.seed_len;
    w.list = nullptr; w.n = 0; w.claim = job.counters + 2; w.n_warps = c.n_warps;
    const WarpLayout WL = warp_layout(c, n);
    char *wb = base + L.warp;
    w.chunks = (uint4 *)(wb + WL.chunks);
    w.chunk_prev = (int32_t *)(wb + WL.chunk_prev);
    w.free_ids = (int32_t *)(wb + WL.free_ids);
    w.aln = (uint64_t *)(wb + WL.aln);
    w.stage = (uint4 *)(wb + WL.stage);
    w.prec = (uint4 *)(wb + WL.prec);
    w.side = (WSide *)(wb + WL.side);
    w.q_ctl = (int32_t *)(wb + WL.q_ctl);
    w.ovq = (int32_t *)(wb + WL.ovq);
    w.n_big = c.n_big; w.big_chunks = c.big_chunks; w.q_wait_ns = c.q_wait_ns;
    w.arena_chunks = c.arena_chunks; w.aln_cap = c.aln_cap;
    w.out_n = job.out_n; w.out_off = job.out_off; w.out_pops = job.out_pops; w.out_trace = job.out_trace;
    w.out_peak = job.out_peak; w.out_fetch = job.out_fetch; w.out_tier = job.out_tier; w.tier = 1;
    w.out_rec = job.out_rec; w.rec_top = job.rec_top; w.rec_cap = job.rec_cap;
    w.ovf = (int32_t *)(base + L.w_ovf); w.ovf_n = job.counters + 3;
    w.dbg = dbg;
    f.n_w_blocks = n_w_blocks;
    GALN_CUDA(cudaMemsetAsync(f.hq, 0xff, (size_t)n * 4, st));
    GALN_CUDA(cudaMemsetAsync(w.ovq, 0xff, (size_t)n * 4, st));
    fused_init_kernel<<<1, 32, 0, st>>>(f.hq_ctl, w.q_ctl, (grid - n_w_blocks) * kFWarps);
    const size_t smem = fused_smem_bytes();
    if (job.occ == kOcc80) {
        if (job.trace) fused_kernel<true, kOcc80><<<grid, kFWarps * 32, smem, st>>>(f);
        else fused_kernel<false, kOcc80><<<grid, kFWarps * 32, smem, st>>>(f);
    } else {
        if (job.trace) fused_kernel<true, kOcc64><<<grid, kFWarps * 32, smem, st>>>(f);
        else fused_kernel<false, kOcc64><<<grid, kFWarps * 32, smem, st>>>(f);
    }
    GALN_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace galn
