// galn_index_files.cpp -- the host side of `galn index`: FASTA records to <prefix>.pac/.ann/.amb, and the
// .bwt/.sa files around the device builder's output (galn_build_index.cu).
//
// Records follow kseq_read() as the reference's src/index/fasta_pac.c:112-170 restates it: a record starts at
// the first '>' or '@' of the input and then at every line start with '>' or '@'; the header's name runs
// to the first white space and, unless that was the line end, the comment to the line end (one final '\r'
// dropped when the comment is longer than one character; an empty comment is "(null)"); the sequence is
// the following lines, one '\r' dropped at a line end by kseq's rule (cr_dropped below). Bases follow
// bwa's bns_fasta2bntseq/add1: A/C/G/T in either case are 0..3, any other byte is ambiguous and becomes
// lrand48() & 3 from srand48(11), drawn in sequence order; runs of the same ambiguous byte are .amb holes.
// FASTQ input (a line starting with '+') is refused.
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <zlib.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <thread>
#include <vector>

#include "galn_aln.h"
#include "galn_host_internal.h"
#include "galn_internal.h"

namespace {

using galn::hvec;

struct Record {
    std::string name, anno;
    int64_t rs = 0, re = 0;            // sequence lines [rs, re) of the input
};

inline bool is_space(int c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

int read_all(const char *path, hvec<uint8_t> &B)
{
    if (FILE *f = fopen(path, "rb")) {            // a plain file: one read of its size
        unsigned char magic[2] = {0, 0};
        const size_t got = fread(magic, 1, 2, f);
        if (!(got == 2 && magic[0] == 0x1f && magic[1] == 0x8b) && fseeko(f, 0, SEEK_END) == 0) {
            const off_t n = ftello(f);
            B.resize(n > 0 ? (size_t)n : 0);
            const bool ok = n >= 0 && fseeko(f, 0, SEEK_SET) == 0 && fread(B.data(), 1, B.size(), f) == B.size();
            fclose(f);
            return ok ? 0 : GALN_EIO;
        }
        fclose(f);
    }
    gzFile fp = gzopen(path, "rb");
    if (!fp) return GALN_EIO;
    gzbuffer(fp, 1 << 20);
    B.clear();
    for (;;) {
        const size_t at = B.size();
        B.resize(at + (4u << 20));
        const int n = gzread(fp, B.data() + at, 4u << 20);
        if (n < 0) { gzclose(fp); return GALN_EIO; }
        B.resize(at + (size_t)n);
        if (n == 0) break;
    }
    return gzclose(fp) == Z_OK ? 0 : GALN_EIO;
}

// whether kseq drops the '\r' at x of a sequence that starts at rs: it cuts one '\r' off the end of a line
// when the sequence read so far is longer than one character; a one-character line at the very end of the
// input is not cut
bool cr_dropped(const uint8_t *B, int64_t N, int64_t x, int64_t rs)
{
    if (x + 1 < N && B[x + 1] != '\n') return false;
    if (x == 0 || B[x - 1] != '\n') return true;
    if (x + 1 == N) return false;
    int64_t y = x - 1;
    while (y >= rs && B[y] == '\n') --y;
    return y >= rs;
}

int parse_records(const hvec<uint8_t> &B, std::vector<Record> &recs)
{
    const int64_t N = (int64_t)B.size();
    int64_t q = 0;
    while (q < N && B[q] != '>' && B[q] != '@') ++q;
    std::vector<int64_t> starts;       // the '>' or '@' of each record
    if (q < N) starts.push_back(q);
    for (int64_t p = q; p + 1 < N; ++p) {
        const uint8_t *nl = (const uint8_t *)memchr(B.data() + p, '\n', N - 1 - p);
        if (!nl) break;
        p = nl - B.data();
        if (B[p + 1] == '>' || B[p + 1] == '@') starts.push_back(p + 1);
        else if (B[p + 1] == '+') return GALN_EINVAL;   // FASTQ
    }
    recs.clear();
    for (size_t i = 0; i < starts.size(); ++i) {
        const int64_t end = i + 1 < starts.size() ? starts[i + 1] : N;
        int64_t p = starts[i] + 1;
        if (p >= N) break;             // the input ends at the '>': kseq gives no record
        Record r;
        int64_t e = p;
        while (e < N && !is_space(B[e])) ++e;
        r.name.assign((const char *)B.data() + p, e - p);
        p = e;
        int c = 0;
        if (p < N) c = B[p++];
        if (c != '\n' && p < N) {
            const uint8_t *nl = (const uint8_t *)memchr(B.data() + p, '\n', N - p);
            const int64_t le = nl ? nl - B.data() : N;
            int64_t l = le - p;
            if (l > 1 && B[le - 1] == '\r') --l;
            if (l > 0) r.anno.assign((const char *)B.data() + p, l);
            p = nl ? le + 1 : N;
        }
        if (r.anno.empty()) r.anno = "(null)";
        r.rs = p < end ? p : end;
        r.re = end;
        recs.push_back(std::move(r));
    }
    return 0;
}

// A piece of one sequence line: input bytes [x, f) go to output offset out.
struct Seg {
    int64_t x, f, out;
};

// the pieces of one record's sequence lines (lines longer than 1 MiB are cut, so threads can share them);
// returns the record's length
int64_t record_segs(const hvec<uint8_t> &B, const Record &r, int64_t out, std::vector<Seg> &segs)
{
    const int64_t start = out, N = (int64_t)B.size();
    int64_t x = r.rs;
    while (x < r.re) {
        const uint8_t *nl = (const uint8_t *)memchr(B.data() + x, '\n', r.re - x);
        const int64_t e = nl ? nl - B.data() : r.re;
        int64_t f = e;
        if (e > x && B[e - 1] == '\r' && cr_dropped(B.data(), N, e - 1, r.rs)) f = e - 1;
        for (int64_t a = x; a < f; a += 1 << 20) {
            const int64_t b = std::min<int64_t>(f, a + (1 << 20));
            segs.push_back(Seg{a, b, out});
            out += b - a;
        }
        x = e + 1;
    }
    return out - start;
}

struct Hole {
    int64_t offset;
    int32_t len;
    char amb;
};

struct Nt4Table {
    uint8_t v[256];
    Nt4Table()
    {
        memset(v, 4, sizeof v);
        const char *b = "ACGT";
        for (int c = 0; c < 4; ++c) v[(uint8_t)b[c]] = v[(uint8_t)b[c] + 32] = (uint8_t)c;
    }
};
const Nt4Table kNt4;

int write_bytes(const std::string &path, const void *p, size_t n)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return GALN_EIO;
    const bool ok = fwrite(p, 1, n, f) == n;
    return (fclose(f) == 0 && ok) ? 0 : GALN_EIO;
}

// body(lo, hi) over [0, n) split among the host's threads
template <class Fn>
void parallel_range(uint64_t n, Fn body)
{
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const uint64_t parts = std::min<uint64_t>(hw, std::max<uint64_t>(1, n >> 20));
    if (parts <= 1) { body((uint64_t)0, n); return; }
    std::vector<std::thread> th;
    for (uint64_t t = 0; t < parts; ++t)
        th.emplace_back(body, n * t / parts, n * (t + 1) / parts);
    for (auto &x : th) x.join();
}

// FASTA -> .pac/.ann/.amb; F = the forward sequence as codes 0..3. The sequence lines of all records are
// listed first; host threads code them, noting the ambiguous bases, which are then replaced in order (their
// lrand48 draws and holes depend only on what came before them).
int fasta_to_pac(const char *fasta, const std::string &prefix, hvec<uint8_t> &F)
{
    hvec<uint8_t> B;
    int rc = read_all(fasta, B);
    if (rc) return rc;
    std::vector<Record> recs;
    rc = parse_records(B, recs);
    if (rc) return rc;
    std::vector<Seg> segs;
    segs.reserve(B.size() / 48 + recs.size() + 16);
    std::vector<int64_t> rec_off(recs.size() + 1);
    int64_t total = 0;
    for (size_t i = 0; i < recs.size(); ++i) {
        rec_off[i] = total;
        total += record_segs(B, recs[i], total, segs);
    }
    rec_off[recs.size()] = total;
    const uint64_t l_pac = (uint64_t)total;
    if (l_pac == 0) return GALN_EINVAL;
    F.resize(l_pac);
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const size_t parts = std::min<size_t>(hw, std::max<size_t>(1, (size_t)(l_pac >> 20)));
    std::vector<std::vector<int64_t>> amb_at(parts);   // position << 8 | the ambiguous byte
    {
        std::vector<std::thread> th;
        for (size_t t = 0; t < parts; ++t)
            th.emplace_back([&, t] {
                const size_t a = segs.size() * t / parts, b = segs.size() * (t + 1) / parts;
                for (size_t k = a; k < b; ++k) {
                    const Seg &g = segs[k];
                    uint8_t *o = F.data() + g.out;
                    for (int64_t j = g.x; j < g.f; ++j) {
                        const uint8_t ch = B[j], c = kNt4.v[ch];
                        o[j - g.x] = c;
                        if (c > 3) amb_at[t].push_back((g.out + (j - g.x)) << 8 | ch);
                    }
                }
            });
        for (auto &x : th) x.join();
    }
    std::vector<Hole> holes;
    std::vector<int> rec_ambs(recs.size());
    uint64_t x = (11ull << 16) | 0x330Eull;          // srand48(11)
    const uint64_t a = 0x5DEECE66Dull, cst = 0xB, m48 = (1ull << 48) - 1;
    size_t r = 0;
    int64_t prev = -2;                                // the last ambiguous base: position << 8 | byte
    for (const auto &v : amb_at)
        for (const int64_t pb : v) {
            const int64_t i = pb >> 8;
            const uint8_t ch = (uint8_t)(pb & 0xff);
            while (rec_off[r + 1] <= i) ++r;
            // the byte before, in the same record, is the same ambiguous byte: the hole goes on
            if (i > rec_off[r] && prev == (((i - 1) << 8) | ch)) ++holes.back().len;
            else {
                holes.push_back(Hole{i, 1, (char)ch});
                ++rec_ambs[r];
            }
            prev = pb;
            x = (a * x + cst) & m48;                 // lrand48() & 3
            F[i] = (uint8_t)((x >> 17) & 3);
        }
    hvec<uint8_t> pac((l_pac + 3) / 4 + 2);
    parallel_range((l_pac + 3) / 4, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t j = lo; j < hi; ++j) {
            uint8_t v = 0;
            for (int k = 0; k < 4; ++k) {
                const uint64_t i = 4 * j + k;
                v |= (uint8_t)((i < l_pac ? F[i] : 0) << (6 - 2 * k));
            }
            pac[j] = v;
        }
    });
    size_t np = (l_pac + 3) / 4;
    if (l_pac % 4 == 0) pac[np++] = 0;
    pac[np++] = (uint8_t)(l_pac % 4);
    rc = write_bytes(prefix + ".pac", pac.data(), np);
    if (rc) return rc;
    std::string ann, amb;
    char line[256];
    snprintf(line, sizeof line, "%llu %d %u\n", (unsigned long long)l_pac, (int)recs.size(), 11u);
    ann += line;
    for (size_t i = 0; i < recs.size(); ++i) {
        ann += "0 " + recs[i].name + " " + recs[i].anno + "\n";
        snprintf(line, sizeof line, "%lld %d %d\n", (long long)rec_off[i], (int)(rec_off[i + 1] - rec_off[i]),
                 rec_ambs[i]);
        ann += line;
    }
    snprintf(line, sizeof line, "%llu %d %u\n", (unsigned long long)l_pac, (int)recs.size(), (unsigned)holes.size());
    amb += line;
    for (const Hole &h : holes) {
        snprintf(line, sizeof line, "%lld %d %c\n", (long long)h.offset, h.len, h.amb);
        amb += line;
    }
    rc = write_bytes(prefix + ".ann", ann.data(), ann.size());
    if (!rc) rc = write_bytes(prefix + ".amb", amb.data(), amb.size());
    return rc;
}

// .bwt: primary, L2[1..4], the body words; .sa: primary, L2[1..4], interval 32, n, the samples
int write_bwt_sa(const std::string &prefix, uint64_t primary, const uint64_t L2[5], const std::vector<uint32_t> &bwt,
                 uint64_t n, const std::vector<uint64_t> &samples)
{
    uint64_t head[7] = {primary, L2[1], L2[2], L2[3], L2[4], 32, n};
    FILE *f = fopen((prefix + ".bwt").c_str(), "wb");
    if (!f) return GALN_EIO;
    bool ok = fwrite(head, 8, 5, f) == 5 && fwrite(bwt.data(), 4, bwt.size(), f) == bwt.size();
    if (fclose(f) != 0 || !ok) return GALN_EIO;
    f = fopen((prefix + ".sa").c_str(), "wb");
    if (!f) return GALN_EIO;
    ok = fwrite(head, 8, 7, f) == 7 && fwrite(samples.data(), 8, samples.size(), f) == samples.size();
    return (fclose(f) == 0 && ok) ? 0 : GALN_EIO;
}

double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int build_text(const uint8_t *fwd, uint64_t l_pac, const std::string &prefix, int device, galn_build_stats *stats,
               double ms_before, int64_t sort_chunk = 0)
{
    for (uint64_t i = 0; i < l_pac; ++i)
        if (fwd[i] > 3) return GALN_EINVAL;
    std::vector<uint32_t> bwt;
    std::vector<uint64_t> samples;
    uint64_t L2[5] = {0, 0, 0, 0, 0}, primary = 0;
    galn_build_stats st{};
    if (cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return GALN_ECUDA; }
    int rc = galn::dev_build_bwt_sa(fwd, l_pac, bwt, L2, primary, samples, &st, sort_chunk);
    if (rc) return rc;
    const double t0 = now_ms();
    rc = write_bwt_sa(prefix, primary, L2, bwt, 2 * l_pac, samples);
    st.ms_files = ms_before + (now_ms() - t0);
    if (stats) *stats = st;
    return rc;
}

}  // namespace

extern "C" int galn_index_build_text(const uint8_t *fwd, uint64_t l_pac, const char *prefix, int device,
                                     galn_build_stats *stats)
{
    if (!fwd || !prefix || l_pac == 0) return GALN_EINVAL;
    return build_text(fwd, l_pac, prefix, device, stats, 0.0);
}

extern "C" int galn_index_build_text_ex(const uint8_t *fwd, uint64_t l_pac, const char *prefix, int device,
                                        int64_t sort_chunk, galn_build_stats *stats)
{
    if (!fwd || !prefix || l_pac == 0 || sort_chunk < 0) return GALN_EINVAL;
    return build_text(fwd, l_pac, prefix, device, stats, 0.0, sort_chunk);
}

extern "C" int galn_fasta_to_pac(const char *fasta, const char *prefix, uint64_t *l_pac)
{
    if (!fasta || !prefix) return GALN_EINVAL;
    hvec<uint8_t> F;
    const int rc = fasta_to_pac(fasta, prefix, F);
    if (!rc && l_pac) *l_pac = F.size();
    return rc;
}

extern "C" int galn_index_build_fasta(const char *fasta, const char *prefix, int device, galn_build_stats *stats)
{
    if (!fasta || !prefix) return GALN_EINVAL;
    const double t0 = now_ms();
    hvec<uint8_t> F;
    int rc = fasta_to_pac(fasta, prefix, F);
    if (rc) return rc;
    return build_text(F.data(), F.size(), prefix, device, stats, now_ms() - t0);
}
