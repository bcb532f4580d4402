// galn_host.cpp -- host side of galn-b200: the C ABI of include/galn_aln.h.
//
//   options       galn_opts_default / galn_opts_parse / galn_cal_maxdiff
//                 (the reference's opt_default, parse_args and aln_cal_maxdiff: src/opt_build.h:23-36,
//                 src/galn.cu:185-250, src/aln_host.c:9-21; this file is compiled with -ffp-contract=off)
//   reads         galn_fastq_read (read_fastq's rules, src/host_io.c:151-205, kseq record semantics)
//   index         galn_index_open (load_bwt, src/host_io.c:29-76) + the device occurrence layout
//   search        galn_aln_run_batch: per-batch options (aln_batch_opt / aln_read_maxdiff,
//                 src/aln_host.c:23-43) and the device tiers (galn_kernels.cu)
//   output        galn_sai_write (src/sai_writer.h:9-21, src/galn.cu:1250-1263)
//   serving       galn_server_* (galn_serve.cpp)
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <ctype.h>
#include <zlib.h>

#include <algorithm>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/galn_aln.h"
#include "galn_internal.h"
#include "galn_host_internal.h"

using namespace galn;

extern "C" const char *galn_version(void) { return "galn-b200 0.1.0 (sm_100a)"; }

// ---------------------------------------------------------------------------------------------------
// options

extern "C" int galn_opts_default(galn_opts *o)
{
    if (!o) return GALN_EINVAL;
    memset(o, 0, sizeof(*o));
    o->s_mm = 3; o->s_gapo = 11; o->s_gape = 4;
    o->max_diff = -1; o->max_gapo = 1; o->max_gape = 6;
    o->indel_end_skip = 5; o->max_del_occ = 10; o->max_entries = 2000000;
    o->mode = 0x01 | 0x02;
    o->seed_len = 32; o->max_seed_diff = 2;
    o->fnr = 0.04f;
    o->n_threads = 1;
    o->max_top2 = 30;
    o->trim_qual = 0;
    return 0;
}

static void set_err(char *err, size_t n, const char *msg, const char *arg)
{
    if (err && n) snprintf(err, n, "%s%s%s", msg, arg ? " " : "", arg ? arg : "");
}

extern "C" int galn_opts_parse(int argc, const char *const *argv, galn_opts *o, const char **pos, int max_pos,
                               int *n_pos, const char **out_path, char *err, size_t err_len)
{
    if (!o) return GALN_EINVAL;
    galn_opts_default(o);
    int opte = -1, np = 0;
    if (out_path) *out_path = nullptr;
    for (int i = 0; i < argc; ++i) {
        const char *a = argv[i];
        const char *v = i + 1 < argc ? argv[i + 1] : nullptr;
        if (a[0] != '-' || !a[1]) {
            if (np < max_pos && pos) pos[np] = a;
            ++np;
            continue;
        }
        if (!strcmp(a, "-L")) { o->mode |= 0x04; continue; }
        if (!strcmp(a, "-N")) { o->mode |= 0x10; o->max_top2 = 0x7fffffff; continue; }
        if (!v) { set_err(err, err_len, "option needs a value:", a); return GALN_EINVAL; }
        if (!strcmp(a, "-n")) {
            if (strchr(v, '.')) { o->fnr = (float)atof(v); o->max_diff = -1; }
            else { o->max_diff = atoi(v); o->fnr = -1.0f; }
        }
        else if (!strcmp(a, "-o")) o->max_gapo = atoi(v);
        else if (!strcmp(a, "-e")) opte = atoi(v);
        else if (!strcmp(a, "-M")) o->s_mm = atoi(v);
        else if (!strcmp(a, "-O")) o->s_gapo = atoi(v);
        else if (!strcmp(a, "-E")) o->s_gape = atoi(v);
        else if (!strcmp(a, "-d")) o->max_del_occ = atoi(v);
        else if (!strcmp(a, "-i")) o->indel_end_skip = atoi(v);
        else if (!strcmp(a, "-l")) o->seed_len = atoi(v);
        else if (!strcmp(a, "-k")) o->max_seed_diff = atoi(v);
        else if (!strcmp(a, "-m")) o->max_entries = atoi(v);
        else if (!strcmp(a, "-dt") || !strcmp(a, "-t")) o->n_threads = atoi(v);
        else if (!strcmp(a, "-R")) o->max_top2 = atoi(v);
        else if (!strcmp(a, "-f")) { if (out_path) *out_path = v; }
        else if (!strcmp(a, "-q")) {
            if (atoi(v) >= 1) { set_err(err, err_len, "-q (quality trimming) is not supported", nullptr); return GALN_EINVAL; }
        }
        else { set_err(err, err_len, "unsupported option", a); return GALN_EINVAL; }
        ++i;
    }
    if (opte > 0) { o->max_gape = opte; o->mode &= ~0x01; }
    if (o->n_threads < 1) o->n_threads = 1;
    if (n_pos) *n_pos = np;
    return 0;
}

extern "C" int galn_cal_maxdiff(int l, double err, double thres)
{
    double elambda = exp(-l * err);
    double sum = elambda, y = 1.0;
    int x = 1;
    for (int k = 1; k < 1000; ++k) {
        y *= l * err;
        x = (int)((unsigned)x * (unsigned)k);   // the reference's int factorial, wrapping
        sum += elambda * y / x;
        if (1.0 - sum < thres) return k;
    }
    return 2;
}

// ---------------------------------------------------------------------------------------------------
// FASTQ / FASTA reading with kseq's record rules

namespace {

// the input as a byte stream, parsed as it arrives; bytes already consumed are dropped from the front of the
// buffer. A gzip input is inflated ahead by a thread of its own (up to four 8 MiB blocks), so inflating and
// parsing overlap; a plain input is read in the parsing thread.
struct Src {
    gzFile fp = nullptr;
    std::vector<unsigned char> buf;
    size_t n = 0, i = 0;
    bool eof = false, err = false;
    // read-ahead of a gzip input
    bool ahead = false;
    std::thread th;
    std::mutex mu;
    std::condition_variable cv_ready, cv_room;
    std::deque<std::vector<unsigned char>> ready;
    std::vector<std::vector<unsigned char>> spare;
    bool done = false, stop = false, ahead_err = false;
    static constexpr size_t kBlock = 8u << 20;
    static constexpr size_t kAhead = 4;

    void start()
    {
        if (!fp || gzdirect(fp)) return;
        ahead = true;
        th = std::thread([this] { inflate_ahead(); });
    }
    void inflate_ahead()
    {
        for (;;) {
            std::vector<unsigned char> b;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_room.wait(lk, [&] { return stop || ready.size() < kAhead; });
                if (stop) return;
                if (!spare.empty()) { b.swap(spare.back()); spare.pop_back(); }
            }
            b.resize(kBlock);
            const int r = gzread(fp, b.data(), (unsigned)b.size());
            std::lock_guard<std::mutex> lk(mu);
            if (r <= 0) {
                ahead_err = r < 0;
                done = true;
                cv_ready.notify_all();
                return;
            }
            b.resize((size_t)r);
            ready.push_back(std::move(b));
            cv_ready.notify_all();
        }
    }
    // stops the read-ahead thread (before gzclose, or when the stream is dropped early)
    void finish()
    {
        if (!ahead) return;
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_room.notify_all();
        th.join();
        ahead = false;
    }
    ~Src() { finish(); }
    bool fill()
    {
        if (eof) return false;
        if (i > 0 && i == n) { n = 0; i = 0; }
        else if (i > (size_t)(16 << 20)) { memmove(buf.data(), buf.data() + i, n - i); n -= i; i = 0; }
        if (!ahead) {
            if (buf.size() - n < (size_t)(4 << 20)) buf.resize(std::max(buf.size() * 2, n + (size_t)(8 << 20)));
            int r = gzread(fp, buf.data() + n, (unsigned)(buf.size() - n));
            if (r < 0) { err = true; eof = true; return false; }
            if (r == 0) { eof = true; return false; }
            n += (size_t)r;
            return true;
        }
        std::vector<unsigned char> b;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_ready.wait(lk, [&] { return !ready.empty() || done; });
            if (ready.empty()) {
                err = ahead_err;
                eof = true;
                return false;
            }
            b = std::move(ready.front());
            ready.pop_front();
        }
        cv_room.notify_all();
        if (buf.size() - n < b.size()) buf.resize(std::max(buf.size() * 2, n + b.size()));
        memcpy(buf.data() + n, b.data(), b.size());
        n += b.size();
        {
            std::lock_guard<std::mutex> lk(mu);
            spare.push_back(std::move(b));
        }
        return true;
    }
    int getc_() { return (i < n || fill()) ? buf[i++] : -1; }
};

// append up to the next '\n' (consumed); drop a trailing '\r' of the whole string when longer than 1
long read_line(Src &s, std::string &t)
{
    if (s.i >= s.n && !s.fill()) return -1;
    for (;;) {
        const unsigned char *p = s.buf.data() + s.i;
        const unsigned char *nl = (const unsigned char *)memchr(p, '\n', s.n - s.i);
        if (nl) {
            t.append((const char *)p, (size_t)(nl - p));
            s.i += (size_t)(nl - p) + 1;
            break;
        }
        t.append((const char *)p, s.n - s.i);
        s.i = s.n;
        if (!s.fill()) break;
    }
    if (t.size() > 1 && t.back() == '\r') t.pop_back();
    return (long)t.size();
}

struct RecordReader {
    int last = 0;
    std::string name, seq, qual;
    // >= 0: sequence length; -1 end of input; -2 malformed record
    int next(Src &s)
    {
        int c;
        if (last == 0) {
            while ((c = s.getc_()) != -1 && c != '>' && c != '@') {}
            if (c == -1) return -1;
            last = c;
        }
        name.clear(); seq.clear(); qual.clear();
        if (s.i >= s.n && !s.fill()) return -1;
        int delim = 0;
        while ((c = s.getc_()) != -1) {
            if (isspace(c)) { delim = c; break; }
            name.push_back((char)c);
        }
        if (delim && delim != '\n') { std::string tmp; read_line(s, tmp); }
        while ((c = s.getc_()) != -1 && c != '>' && c != '+' && c != '@') {
            if (c == '\n') continue;
            seq.push_back((char)c);
            read_line(s, seq);
        }
        if (c == '>' || c == '@') last = c;
        if (c != '+') return (int)seq.size();
        while ((c = s.getc_()) != -1 && c != '\n') {}
        if (c == -1) return -2;
        while (read_line(s, qual) >= 0 && qual.size() < seq.size()) {}
        last = 0;
        if (seq.size() != qual.size()) return -2;
        return (int)seq.size();
    }
};

struct ReadSetPriv {
    std::vector<char> seq;
    std::vector<int64_t> off;
    std::vector<int32_t> batch;
    std::vector<std::string> names;
    std::vector<char *> name_ptrs;
    void publish(galn_read_set *out)
    {
        name_ptrs.resize(names.size());
        for (size_t i = 0; i < names.size(); ++i) name_ptrs[i] = (char *)names[i].c_str();
        out->reads.n_reads = (int32_t)batch.size();
        out->reads.seq = seq.data();
        out->reads.offset = off.data();
        out->reads.batch = batch.data();
        out->names = name_ptrs.data();
        out->_priv = this;
    }
};

}  // namespace

// An open input: the record reader and the bwa batch it is in (read_fastq's rules, src/host_io.c:151-205:
// 0x40000 reads per batch, empty reads skipped, a malformed record dropped and ending its batch, and ending
// the input when it comes first in a batch).
struct galn_fastq_stream {
    Src src;
    RecordReader rr;
    int batch = 0;
    bool done = false;
};

// Appends the records of the current batch to P (batch ids as in the whole input); false when the input is
// done. Stops at the batch's end.
static bool stream_batch(galn_fastq_stream *st, ReadSetPriv *P)
{
    if (st->done) return false;
    int in_batch = 0;
    for (;;) {
        int l = st->rr.next(st->src);
        if (l < 0) {
            if (in_batch == 0 || l == -1) { st->done = true; return in_batch > 0; }
            ++st->batch;                // a malformed record ends the batch
            return true;
        }
        if (st->rr.seq.empty()) continue;  // empty reads are skipped
        P->seq.insert(P->seq.end(), st->rr.seq.begin(), st->rr.seq.end());
        P->off.push_back((int64_t)P->seq.size());
        P->batch.push_back(st->batch);
        P->names.push_back(st->rr.name);
        if (++in_batch == kBatchReads) { ++st->batch; return true; }
    }
}

extern "C" galn_fastq_stream *galn_fastq_open(const char *path, int *err)
{
    if (!path) { if (err) *err = GALN_EINVAL; return nullptr; }
    gzFile fp = gzopen(path, "rb");
    if (!fp) { if (err) *err = GALN_EIO; return nullptr; }
    gzbuffer(fp, 1 << 20);
    auto *st = new galn_fastq_stream();
    st->src.fp = fp;
    st->src.start();
    if (err) *err = 0;
    return st;
}

extern "C" int galn_fastq_next(galn_fastq_stream *st, galn_read_set *out)
{
    if (!st || !out) return GALN_EINVAL;
    memset(out, 0, sizeof(*out));
    auto *P = new ReadSetPriv();
    P->off.push_back(0);
    stream_batch(st, P);
    if (st->src.err) { delete P; return GALN_EIO; }
    P->publish(out);
    return 0;
}

extern "C" int galn_fastq_close(galn_fastq_stream *st)
{
    if (!st) return GALN_EINVAL;
    st->src.finish();
    int rc = st->src.fp && gzclose(st->src.fp) != Z_OK ? GALN_EIO : 0;
    delete st;
    return rc;
}

extern "C" int galn_fastq_read(const char *path, galn_read_set *out)
{
    if (!path || !out) return GALN_EINVAL;
    memset(out, 0, sizeof(*out));
    int e = 0;
    galn_fastq_stream *st = galn_fastq_open(path, &e);
    if (!st) return e;
    auto *P = new ReadSetPriv();
    P->off.push_back(0);
    while (stream_batch(st, P)) {}
    const bool bad = st->src.err;
    const int rc = galn_fastq_close(st);
    if (bad || rc) { delete P; return GALN_EIO; }
    P->publish(out);
    return 0;
}

extern "C" int galn_read_set_free(galn_read_set *rs)
{
    if (!rs) return GALN_EINVAL;
    delete (ReadSetPriv *)rs->_priv;
    memset(rs, 0, sizeof(*rs));
    return 0;
}

// ---------------------------------------------------------------------------------------------------
// index

static galn_index *index_from_words(const uint64_t hdr[5], const uint32_t *body, uint64_t n_words, int device, int *err)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || device < 0 || device >= ndev) {
        cudaGetLastError();
        if (err) *err = GALN_ECUDA;
        return nullptr;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
        if (err) *err = GALN_ECUDA;
        return nullptr;
    }
    auto *ix = new galn_index();
    DevIndex &d = ix->dev;
    d.device = device;
    d.primary = hdr[0];
    d.L2[0] = 0;
    for (int c = 0; c < 4; ++c) d.L2[c + 1] = hdr[c + 1];
    d.seq_len = d.L2[4];
    uint64_t nb = (d.seq_len + 127) / 128;
    uint64_t expect = 8 * (nb + 1) + (d.seq_len + 15) / 16;
    if (d.seq_len == 0 || n_words != expect || d.primary == 0 || d.primary > d.seq_len) {
        delete ix;
        if (err) *err = GALN_EIO;
        return nullptr;
    }
    ix->sms = prop.multiProcessorCount;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ix->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ix;
        if (err) *err = GALN_ECUDA;
        return nullptr;
    }
    ix->main.stream = ix->stream;
    int rc = dev_index_build(d, body, n_words, ix->stream);
    if (rc) {
        dev_index_free(d);
        delete ix;
        if (err) *err = rc;
        return nullptr;
    }
    galn::index_l2_policy(ix, ix->stream, ix->occ);
    ix->main.l2_occ = ix->occ;
    if (err) *err = 0;
    return ix;
}

// Keep the occurrence blocks in L2: a persisting access-policy window over them on every stream that
// searches (the set-aside is a limit of this process's context and ends with it). The search reads the
// index at random on every step, while stack pushes and pops stream through; without the window the
// stream evicts the index.
void galn::index_l2_policy(galn_index *ix, cudaStream_t st, int occ)
{
    const void *blocks = occ == 80 ? ix->dev.blocks80 : ix->dev.blocks;
    const uint64_t n_blocks = occ == 80 ? ix->dev.n_blocks80 : ix->dev.n_blocks;
    if (!ix->l2_persist || !blocks) return;
    int maxw = 0, maxp = 0;
    cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, ix->dev.device);
    cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, ix->dev.device);
    if (maxw <= 0 || maxp <= 0) return;
    const size_t bytes = std::min<size_t>((size_t)n_blocks * 32, (size_t)maxw);
    const size_t persist = std::min<size_t>(bytes, (size_t)maxp);
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, persist) != cudaSuccess) { cudaGetLastError(); return; }
    cudaStreamAttrValue v;
    memset(&v, 0, sizeof(v));
    v.accessPolicyWindow.base_ptr = const_cast<void *>(blocks);
    v.accessPolicyWindow.num_bytes = bytes;
    v.accessPolicyWindow.hitRatio = (float)std::min(1.0, (double)persist / (double)bytes);
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    if (cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &v) != cudaSuccess) cudaGetLastError();
}

// With the whole index inside the persisting window, read it once through L2 in a coalesced pass before a
// search: after other traffic (the reads' upload, another job) the first tier would otherwise bring it back
// by random 32-byte misses, each costing a DRAM burst. Returns the launches made (0 or 1), or < 0 on error.
int galn::index_l2_warm(galn_index *ix, cudaStream_t st, int occ)
{
    const void *blocks = occ == 80 ? ix->dev.blocks80 : ix->dev.blocks;
    const uint64_t n_blocks = occ == 80 ? ix->dev.n_blocks80 : ix->dev.n_blocks;
    if (!ix->l2_persist || !blocks || !ix->l2_warm) return 0;
    int maxw = 0, maxp = 0;
    cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, ix->dev.device);
    cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, ix->dev.device);
    const size_t bytes = (size_t)n_blocks * 32;
    if (maxw <= 0 || maxp <= 0 || bytes > (size_t)maxw || bytes > (size_t)maxp) return 0;
    const int rc = dev_l2_warm(blocks, bytes, ix->dev.device, st);
    return rc ? rc : 1;
}

void galn::index_l2_clear(galn_index *ix, cudaStream_t st)
{
    cudaStreamAttrValue v;
    memset(&v, 0, sizeof(v));
    v.accessPolicyWindow.num_bytes = 0;
    if (cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &v) != cudaSuccess) cudaGetLastError();
}

extern "C" galn_index *galn_index_open(const char *prefix, int device, int *err)
{
    if (!prefix) { if (err) *err = GALN_EINVAL; return nullptr; }
    std::string fn = std::string(prefix) + ".bwt";
    FILE *fp = fopen(fn.c_str(), "rb");
    if (!fp) { if (err) *err = GALN_EIO; return nullptr; }
    uint64_t hdr[5];
    if (fread(hdr, 8, 5, fp) != 5) { fclose(fp); if (err) *err = GALN_EIO; return nullptr; }
    fseeko(fp, 0, SEEK_END);
    long long sz = ftello(fp);
    fseeko(fp, 40, SEEK_SET);
    if (sz < 40 || (sz - 40) % 4) { fclose(fp); if (err) *err = GALN_EIO; return nullptr; }
    uint64_t n_words = (uint64_t)(sz - 40) / 4;
    uint32_t *body = nullptr;
    if (cudaMallocHost(&body, n_words * 4 + 4) != cudaSuccess) { fclose(fp); if (err) *err = GALN_ENOMEM; return nullptr; }
    size_t got = 0;
    while (got < n_words) {
        size_t r = fread(body + got, 4, std::min<size_t>(n_words - got, (size_t)1 << 26), fp);
        if (r == 0) break;
        got += r;
    }
    fclose(fp);
    if (got != n_words) { cudaFreeHost(body); if (err) *err = GALN_EIO; return nullptr; }
    galn_index *ix = index_from_words(hdr, body, n_words, device, err);
    cudaFreeHost(body);
    return ix;
}

extern "C" galn_index *galn_index_open_mem(const void *bytes, size_t n_bytes, int device, int *err)
{
    if (!bytes || n_bytes < 40 || (n_bytes - 40) % 4) { if (err) *err = GALN_EINVAL; return nullptr; }
    uint64_t hdr[5];
    memcpy(hdr, bytes, 40);
    return index_from_words(hdr, (const uint32_t *)((const char *)bytes + 40), (n_bytes - 40) / 4, device, err);
}

extern "C" int galn_index_close(galn_index *ix)
{
    if (!ix) return GALN_EINVAL;
    cudaSetDevice(ix->dev.device);
    ix->main.release();
    galn::Buf *sa[] = {&ix->sa_samples, &ix->sa_k, &ix->sa_len, &ix->sa_pos, &ix->sa_strand};
    for (Buf *b : sa) b->release();
    dev_index_free(ix->dev);
    if (ix->stream) cudaStreamDestroy(ix->stream);
    delete ix;
    return 0;
}

// ---------------------------------------------------------------------------------------------------
// suffix-array positions (samse's coordinate step)

extern "C" int galn_index_load_sa(galn_index *ix, const char *prefix)
{
    if (!ix || !prefix) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    // bwt_restore_sa (bwa's bwt.c:421-441): primary, 4 counts (skipped), interval, seq_len, then the samples
    // of rows intv, 2 intv, ...; row 0 (the $ row) is -1
    const std::string fn = std::string(prefix) + ".sa";
    FILE *fp = fopen(fn.c_str(), "rb");
    if (!fp) return GALN_EIO;
    uint64_t hdr[7];
    if (fread(hdr, 8, 7, fp) != 7) { fclose(fp); return GALN_EIO; }
    const uint64_t primary = hdr[0], intv = hdr[5], seq_len = hdr[6];
    if (primary != ix->dev.primary || seq_len != ix->dev.seq_len || intv == 0 || (intv & (intv - 1))) {
        fclose(fp);
        return GALN_EIO;
    }
    const uint64_t n_sa = (seq_len + intv) / intv;
    std::vector<uint64_t> sa((size_t)n_sa);
    sa[0] = ~0ull;
    const size_t got = n_sa > 1 ? fread(sa.data() + 1, 8, (size_t)(n_sa - 1), fp) : 0;
    fclose(fp);
    if (got != n_sa - 1) return GALN_EIO;
    if (cudaSetDevice(ix->dev.device) != cudaSuccess) return GALN_ECUDA;
    if (ix->sa_samples.ensure((size_t)n_sa * 8)) return GALN_ENOMEM;
    if (cudaMemcpy(ix->sa_samples.p, sa.data(), (size_t)n_sa * 8, cudaMemcpyHostToDevice) != cudaSuccess) return GALN_ECUDA;
    ix->sa_intv = intv;
    ix->n_sa = n_sa;
    return 0;
}

static int sa_query(galn_index *ix, const uint64_t *rows, const int32_t *ref_len, int64_t n, uint64_t *pos, int8_t *strand)
{
    if (!ix || n < 0 || (n > 0 && (!rows || !pos || (ref_len && !strand)))) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    if (!ix->n_sa) return GALN_EINVAL;                 // galn_index_load_sa first
    if (n == 0) return 0;
    if (cudaSetDevice(ix->dev.device) != cudaSuccess) return GALN_ECUDA;
    const size_t nn = (size_t)n;
    if (ix->sa_k.ensure(nn * 8) || ix->sa_pos.ensure(nn * 8) || (ref_len && (ix->sa_len.ensure(nn * 4) ||
                                                                               ix->sa_strand.ensure(nn))))
        return GALN_ENOMEM;
    cudaStream_t st = ix->stream;
    if (cudaMemcpyAsync(ix->sa_k.p, rows, nn * 8, cudaMemcpyHostToDevice, st) != cudaSuccess) return GALN_ECUDA;
    if (ref_len && cudaMemcpyAsync(ix->sa_len.p, ref_len, nn * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return GALN_ECUDA;
    int rc = galn::dev_sa_walk(ix->dev, (const uint64_t *)ix->sa_samples.p, ix->sa_intv, (const uint64_t *)ix->sa_k.p, n,
                               ref_len ? (const int32_t *)ix->sa_len.p : nullptr, (uint64_t *)ix->sa_pos.p,
                               ref_len ? (int8_t *)ix->sa_strand.p : nullptr, st);
    if (rc) return rc;
    if (cudaMemcpyAsync(pos, ix->sa_pos.p, nn * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess) return GALN_ECUDA;
    if (ref_len && cudaMemcpyAsync(strand, ix->sa_strand.p, nn, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return GALN_ECUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? 0 : GALN_ECUDA;
}

extern "C" int galn_bwt_sa(galn_index *ix, const uint64_t *rows, int64_t n, uint64_t *sa)
{
    return sa_query(ix, rows, nullptr, n, sa, nullptr);
}

extern "C" int galn_sa2pos(galn_index *ix, const uint64_t *rows, const int32_t *ref_len, int64_t n, uint64_t *pos,
                           int8_t *strand)
{
    if (!ref_len) return GALN_EINVAL;
    return sa_query(ix, rows, ref_len, n, pos, strand);
}

extern "C" int galn_index_occ(galn_index *ix, int layout, const uint64_t *rows, int64_t n, uint64_t *occ, uint32_t *fetch)
{
    if (!ix || n < 0 || (layout != 64 && layout != 80) || (n > 0 && (!rows || !occ))) return GALN_EINVAL;
    std::lock_guard<std::mutex> lk(ix->mu);
    if (n == 0) return 0;
    for (int64_t i = 0; i < n; ++i)
        if (rows[i] != ~0ull && rows[i] > ix->dev.seq_len) return GALN_EINVAL;
    if (cudaSetDevice(ix->dev.device) != cudaSuccess) return GALN_ECUDA;
    const size_t nn = (size_t)n;
    void *d = nullptr;
    const size_t o_occ = (nn * 8 + 255) & ~(size_t)255, o_f = o_occ + nn * 32;
    if (cudaMalloc(&d, o_f + nn * 4) != cudaSuccess) { cudaGetLastError(); return GALN_ENOMEM; }
    cudaStream_t st = ix->stream;
    char *b = (char *)d;
    int rc = 0;
    if (cudaMemcpyAsync(b, rows, nn * 8, cudaMemcpyHostToDevice, st) != cudaSuccess) rc = GALN_ECUDA;
    if (!rc) rc = galn::dev_occ_probe(ix->dev, layout, (const uint64_t *)b, n, (uint64_t *)(b + o_occ),
                                      (uint32_t *)(b + o_f), st);
    if (!rc && cudaMemcpyAsync(occ, b + o_occ, nn * 32, cudaMemcpyDeviceToHost, st) != cudaSuccess) rc = GALN_ECUDA;
    if (!rc && fetch && cudaMemcpyAsync(fetch, b + o_f, nn * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) rc = GALN_ECUDA;
    if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = GALN_ECUDA;
    cudaFree(d);
    return rc;
}

extern "C" int galn_index_info(const galn_index *ix, uint64_t *seq_len, uint64_t *primary, uint64_t *device_bytes)
{
    if (!ix) return GALN_EINVAL;
    if (seq_len) *seq_len = ix->dev.seq_len;
    if (primary) *primary = ix->dev.primary;
    if (device_bytes) *device_bytes = ix->dev.n_blocks * 32;
    return 0;
}

// ---------------------------------------------------------------------------------------------------
// results and .sai

extern "C" int galn_results_free(galn_results *res)
{
    if (!res) return GALN_EINVAL;
    delete (ResultsPriv *)res->_priv;
    memset(res, 0, sizeof(*res));
    return 0;
}

// an open .sai stream: the header is written at open, then the reads of each appended result set
struct galn_sai_writer {
    FILE *fp = nullptr;
    bool own = false;
    int err = 0;                        // 4: a read with an error code was written with 0 records; 5: I/O
    std::vector<char> buf;
    void put(const void *p, size_t n)
    {
        buf.insert(buf.end(), (const char *)p, (const char *)p + n);
        if (buf.size() >= (1 << 20)) flush();
    }
    void flush()
    {
        if (!buf.empty() && fwrite(buf.data(), 1, buf.size(), fp) != buf.size()) err = 5;
        buf.clear();
    }
};

extern "C" galn_sai_writer *galn_sai_open(const char *path, const galn_opts *o, int *err)
{
    static_assert(sizeof(galn_opts) == 64, "gap_opt_t is 64 bytes");
    static_assert(sizeof(galn_aln1) == 24, "bwt_aln1_t is 24 bytes");
    if (!o) { if (err) *err = GALN_EINVAL; return nullptr; }
    FILE *fp = path ? fopen(path, "wb") : stdout;
    if (!fp) { if (err) *err = 5; return nullptr; }
    auto *w = new galn_sai_writer();
    w->fp = fp;
    w->own = path != nullptr;
    w->buf.reserve(1 << 20);
    w->put("SAI\1", 4);
    w->put(o, sizeof(*o));
    if (err) *err = 0;
    return w;
}

extern "C" int galn_sai_append(galn_sai_writer *w, const galn_results *res)
{
    if (!w || !res) return GALN_EINVAL;
    for (int r = 0; r < res->n_reads; ++r) {
        int32_t na = res->n_aln[r];
        if (na < 0) { if (!w->err) w->err = 4; na = 0; }
        w->put(&na, 4);
        if (na > 0) w->put(res->rec + res->rec_offset[r], (size_t)na * sizeof(galn_aln1));
    }
    return w->err == 5 ? 5 : 0;
}

extern "C" int galn_sai_close(galn_sai_writer *w)
{
    if (!w) return GALN_EINVAL;
    w->flush();
    if (fflush(w->fp) != 0 || ferror(w->fp)) w->err = 5;
    if (w->own && fclose(w->fp) != 0) w->err = 5;
    const int err = w->err;
    delete w;
    return err;
}

extern "C" int galn_sai_write(const char *path, const galn_opts *o, const galn_results *res)
{
    if (!o || !res) return GALN_EINVAL;
    int e = 0;
    galn_sai_writer *w = galn_sai_open(path, o, &e);
    if (!w) return e;
    galn_sai_append(w, res);
    return galn_sai_close(w);
}
