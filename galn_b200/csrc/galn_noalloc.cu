// galn_noalloc.cu -- galn_aln_run_noalloc: the first-tier search without any device allocation.
//
// Some callers cannot allocate device memory while they run the search: a host framework that owns the
// GPU's memory through its own pool and forbids outside cudaMalloc/cudaFree, code running inside a
// memory budget that must not grow, or a pipeline stage that must not synchronise the device (cudaFree
// does). For them this entry point takes every input and output as the caller's own device buffers and
// keeps all of its scratch (per-thread stacks, bucket heads, width arrays, the encoded reads and the work
// counter) in one file-scope __device__ array of kScratchBytes. That array belongs to the library: every
// GPU that loads the library holds it until the process exits. The per-length max_diff table travels in the
// kernel's parameters, so the only stream operations of a call are one memset of the counter and the launch.
//
// Host code never passes g_scratch itself to a kernel: in host code the name is only a stand-in for the
// symbol, not a device address. The device address is looked up once per device with
// cudaGetSymbolAddress, the first time the entry point runs on that device (with that device current);
// that first call should therefore come before any stream capture. All calls share the one array and it
// keeps the last call's contents, so the counter is cleared at the start of every call, and calls that
// overlap on the GPU (on different streams, or from several host threads) race on it: serialise them.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "galn_host_internal.h"
#include "galn_search.cuh"

namespace galn {
namespace {

constexpr size_t kScratchBytes = (size_t)32 << 20;     // 32 MiB of scratch per device
constexpr int kNaMaxLen = 1024;                        // longest read this entry point takes
constexpr int kNaMaxStacks = 512;                      // most score buckets
constexpr int kNaMaxRec = 256;                         // most records per read
constexpr int kNaCap = 2048;                           // stack entries per thread (bump-allocated)
constexpr size_t kHdr = 256;                           // work counter

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
void *g_addr[64];

__host__ __device__ inline size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

struct NaArgs {
    IndexView ix;
    BatchOpt bo;
    const char *seq;
    const int64_t *off;
    int n, max_len, seed_len, n_slots, rec_per_read;
    int32_t *n_aln;
    uint64_t *rec;
    unsigned char *scratch;           // device address of g_scratch
    size_t slot_bytes;
    Workspace ws;                     // arrays inside the scratch (strided by slot)
    size_t q_off;                     // offset of the per-slot query buffers inside the scratch
    size_t q_stride;                  // bytes per slot's query buffer
    int16_t md[kNaMaxLen + 1];        // max_diff by read length (bwa_cal_maxdiff, computed on the host)
};

__global__ void __launch_bounds__(128) noalloc_kernel(const __grid_constant__ NaArgs a)
{
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= a.n_slots) return;
    int32_t *claim = (int32_t *)a.scratch;
    uint8_t *q = a.scratch + a.q_off + (size_t)slot * a.q_stride;
    for (;;) {
        int r = atomicAdd(claim, 1);
        if (r >= a.n) break;
        const int64_t s = a.off[r];
        const int64_t len64 = a.off[r + 1] - s;
        if (len64 < 0 || len64 > a.max_len) { a.n_aln[r] = -20; continue; }   // GALN_EINVAL for this read
        const int len = (int)len64;
        for (int j = 0; j < len; ++j) {   // reverse, complement; anything but ACGT is ambiguous
            uint8_t b;
            switch (a.seq[s + len - 1 - j] | 0x20) {
            case 'a': b = 3; break;
            case 'c': b = 2; break;
            case 'g': b = 1; break;
            case 't': b = 0; break;
            default: b = 4;
            }
            q[j] = b;
        }
        uint64_t *W = a.ws.wid + (size_t)slot * a.ws.wcap;
        uint64_t *SW = W + (len + 1);
        const bool use_seed = len > a.seed_len;
        uint32_t fetches = 0;
        cal_width(a.ix, len, q, W, fetches);
        if (use_seed) cal_width(a.ix, a.seed_len, q + (len - a.seed_len), SW, fetches);
        SearchResult R = match_gap<false, false, false>(a.ix, a.bo, (int)a.md[len], len, q, W, SW, use_seed, a.ws, slot,
                                                        fetches);
        if (R.ret > 0) {
            const uint64_t *src = a.ws.aln + (size_t)slot * a.ws.aln_cap * 3;
            uint64_t *dst = a.rec + (size_t)r * a.rec_per_read * 3;
            for (int j = 0; j < 3 * R.ret; ++j) dst[j] = src[j];
        }
        a.n_aln[r] = R.ret;
    }
}

}  // namespace
}  // namespace galn

using namespace galn;

extern "C" int galn_aln_run_noalloc(galn_index *ix, const galn_opts *o, int32_t n_reads, int32_t max_len,
                                    const char *d_seq, const int64_t *d_offset, int32_t *d_n_aln, galn_aln1 *d_rec,
                                    int32_t rec_per_read, void *stream)
{
    if (!ix || !o || n_reads < 0 || n_reads > kBatchReads) return GALN_EINVAL;
    if (max_len < 0 || max_len > kNaMaxLen || rec_per_read < 1 || rec_per_read > kNaMaxRec) return GALN_EINVAL;
    if (n_reads > 0 && (!d_seq || !d_offset || !d_n_aln || !d_rec)) return GALN_EINVAL;
    if (o->s_mm < 0 || o->s_gapo < 0 || o->s_gape < 0) return GALN_EINVAL;
    if (ix->dev.seq_len >= (1ull << 38)) return GALN_EINVAL;
    // the batch's options (all reads are one bwa batch) and each length's max_diff, on the host
    BatchOpt bo;
    memset(&bo, 0, sizeof(bo));
    bo.s_mm = o->s_mm; bo.s_gapo = o->s_gapo; bo.s_gape = o->s_gape; bo.mode = o->mode;
    bo.indel_end_skip = o->indel_end_skip; bo.max_del_occ = o->max_del_occ; bo.max_entries = o->max_entries;
    bo.max_diff = o->max_diff; bo.max_gapo = o->max_gapo; bo.max_gape = o->max_gape;
    bo.max_seed_diff = o->max_seed_diff; bo.seed_len = o->seed_len; bo.max_top2 = o->max_top2;
    if (o->fnr > 0.0) bo.max_diff = galn_cal_maxdiff(max_len, 0.02, o->fnr);
    if (bo.max_diff < bo.max_gapo) bo.max_gapo = bo.max_diff;
    bo.n_stacks = (bo.max_diff + 1) * bo.s_mm + (bo.max_gapo + 1) * bo.s_gapo + (bo.max_gape + 1) * bo.s_gape;
    if (bo.n_stacks > kNaMaxStacks || bo.max_gapo > 126 || bo.max_gape > 126) return GALN_EINVAL;
    if (n_reads == 0) return 0;
    const int seed_len = o->seed_len < 0 ? 0 : o->seed_len;
    const int wcap = max_len + 1 + (max_len > seed_len ? seed_len + 1 : 0) + 1;
    const int hcap = bo.n_stacks > 0 ? bo.n_stacks : 1;
    // per-slot strides exactly as match_gap indexes them (cap, hcap, wcap, aln_cap elements)
    const size_t st_ent = (size_t)kNaCap * 16, st_link = (size_t)kNaCap * 4, st_heads = (size_t)hcap * 4,
                 st_wid = (size_t)wcap * 8, st_aln = (size_t)rec_per_read * 24, st_q = a256((size_t)max_len + 1);
    const size_t slot_bytes = st_ent + st_link + st_heads + st_wid + st_aln + st_q + 6 * 256;
    const size_t fixed = kHdr;
    const int n_slots = (int)std::min<size_t>((size_t)n_reads, (kScratchBytes - fixed) / slot_bytes);
    if (n_slots < 1) return GALN_EINVAL;

    std::lock_guard<std::mutex> lk(g_mu);
    const int dev = ix->dev.device;
    if (dev < 0 || dev >= 64) return GALN_EINVAL;
    int prev_dev = 0;
    if (cudaGetDevice(&prev_dev) != cudaSuccess) return GALN_ECUDA;
    if (cudaSetDevice(dev) != cudaSuccess) return GALN_ECUDA;
    int rc = 0;
    cudaStream_t st = (cudaStream_t)stream;
    do {
        if (!g_addr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) { rc = GALN_ECUDA; break; }
            g_addr[dev] = p;
        }
        unsigned char *base = (unsigned char *)g_addr[dev];
        NaArgs a;
        memset(&a, 0, sizeof(a));
        for (int L = 0; L <= max_len && !rc; ++L) {
            const int md = o->fnr > 0.0 ? galn_cal_maxdiff(L, 0.02, o->fnr) : bo.max_diff;
            if (md < -32768 || md > 125) rc = GALN_EINVAL;
            else a.md[L] = (int16_t)md;
        }
        if (rc) break;
        if (cudaMemsetAsync(base, 0, kHdr, st) != cudaSuccess) { rc = GALN_ECUDA; break; }
        a.ix.blk = (const uint4 *)ix->dev.blocks;
        a.ix.primary = ix->dev.primary;
        a.ix.seq_len = ix->dev.seq_len;
        for (int c = 0; c < 4; ++c) a.ix.C[c] = ix->dev.L2[c];
        memcpy(a.ix.sb, ix->dev.sb, sizeof(a.ix.sb));
        a.bo = bo;
        a.seq = d_seq; a.off = d_offset; a.n = n_reads; a.max_len = max_len; a.seed_len = seed_len;
        a.n_slots = n_slots; a.rec_per_read = rec_per_read;
        a.n_aln = d_n_aln; a.rec = (uint64_t *)d_rec;
        a.scratch = base;
        size_t off = fixed, ns = (size_t)n_slots;
        a.ws.ent = (uint4 *)(base + off);         off += a256(ns * st_ent);
        a.ws.link = (int32_t *)(base + off);      off += a256(ns * st_link);
        a.ws.heads = (int32_t *)(base + off);     off += a256(ns * st_heads);
        a.ws.wid = (uint64_t *)(base + off);      off += a256(ns * st_wid);
        a.ws.aln = (uint64_t *)(base + off);      off += a256(ns * st_aln);
        a.q_off = off;                            off += a256(ns * st_q);
        a.q_stride = st_q;
        if (off > kScratchBytes) { rc = GALN_EINVAL; break; }
        a.ws.cap = kNaCap; a.ws.hcap = hcap; a.ws.wcap = wcap; a.ws.aln_cap = rec_per_read;
        noalloc_kernel<<<(n_slots + 127) / 128, 128, 0, st>>>(a);
        if (cudaGetLastError() != cudaSuccess) { rc = GALN_ECUDA; break; }
    } while (0);
    cudaSetDevice(prev_dev);
    return rc;
}
