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

#include <chrono>
#include <string>
#include <vector>

#include "galn_aln.h"
#include "galn_internal.h"

namespace {

struct Record {
    std::string name, anno;
    int64_t rs = 0, re = 0;            // sequence lines [rs, re) of the input
};

inline bool is_space(int c) { return c == ' ' || (c >= '\t' && c <= '\r'); }

int read_all(const char *path, std::vector<uint8_t> &B)
{
    gzFile fp = gzopen(path, "rb");
    if (!fp) return GALN_EIO;
    gzbuffer(fp, 1 << 20);
    B.clear();
    std::vector<uint8_t> chunk(1 << 22);
    for (;;) {
        const int n = gzread(fp, chunk.data(), (unsigned)chunk.size());
        if (n < 0) { gzclose(fp); return GALN_EIO; }
        if (n == 0) break;
        B.insert(B.end(), chunk.begin(), chunk.begin() + n);
    }
    return gzclose(fp) == Z_OK ? 0 : GALN_EIO;
}

// whether kseq drops the '\r' at x of a sequence that starts at rs: it cuts one '\r' off the end of a line
// when the sequence read so far is longer than one character; a one-character line at the very end of the
// input is not cut
bool cr_dropped(const std::vector<uint8_t> &B, int64_t x, int64_t rs)
{
    const int64_t N = (int64_t)B.size();
    if (x + 1 < N && B[x + 1] != '\n') return false;
    if (x == 0 || B[x - 1] != '\n') return true;
    if (x + 1 == N) return false;
    int64_t y = x - 1;
    while (y >= rs && B[y] == '\n') --y;
    return y >= rs;
}

int parse_records(const std::vector<uint8_t> &B, std::vector<Record> &recs)
{
    const int64_t N = (int64_t)B.size();
    int64_t q = 0;
    while (q < N && B[q] != '>' && B[q] != '@') ++q;
    std::vector<int64_t> starts;       // the '>' or '@' of each record
    if (q < N) starts.push_back(q);
    for (int64_t p = q; p + 1 < N; ++p) {
        if (B[p] != '\n') continue;
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

// one record's sequence bytes
void record_seq(const std::vector<uint8_t> &B, const Record &r, std::string &out)
{
    out.clear();
    int64_t x = r.rs;
    while (x < r.re) {
        const uint8_t *nl = (const uint8_t *)memchr(B.data() + x, '\n', r.re - x);
        const int64_t e = nl ? nl - B.data() : r.re;
        int64_t f = e;
        if (e > x && B[e - 1] == '\r' && cr_dropped(B, e - 1, r.rs)) f = e - 1;
        out.append((const char *)B.data() + x, f - x);
        x = e + 1;
    }
}

struct Hole {
    int64_t offset;
    int32_t len;
    char amb;
};

int nt4(uint8_t c)
{
    switch (c) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return 4;
    }
}

int write_bytes(const std::string &path, const void *p, size_t n)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return GALN_EIO;
    const bool ok = fwrite(p, 1, n, f) == n;
    return (fclose(f) == 0 && ok) ? 0 : GALN_EIO;
}

// FASTA -> .pac/.ann/.amb; F = the forward sequence as codes 0..3
int fasta_to_pac(const char *fasta, const std::string &prefix, std::vector<uint8_t> &F)
{
    std::vector<uint8_t> B;
    int rc = read_all(fasta, B);
    if (rc) return rc;
    std::vector<Record> recs;
    rc = parse_records(B, recs);
    if (rc) return rc;
    F.clear();
    std::vector<Hole> holes;
    std::vector<int64_t> rec_len(recs.size()), rec_off(recs.size());
    std::vector<int> rec_ambs(recs.size());
    uint64_t x = (11ull << 16) | 0x330Eull;          // srand48(11)
    const uint64_t a = 0x5DEECE66Dull, cst = 0xB, m48 = (1ull << 48) - 1;
    std::string seq;
    for (size_t i = 0; i < recs.size(); ++i) {
        record_seq(B, recs[i], seq);
        rec_off[i] = (int64_t)F.size();
        rec_len[i] = (int64_t)seq.size();
        int last = 0;
        for (size_t j = 0; j < seq.size(); ++j) {
            const uint8_t ch = (uint8_t)seq[j];
            int c = nt4(ch);
            if (c >= 4) {
                if (last == ch) ++holes.back().len;
                else {
                    holes.push_back(Hole{rec_off[i] + (int64_t)j, 1, (char)ch});
                    ++rec_ambs[i];
                }
                x = (a * x + cst) & m48;             // lrand48() & 3
                c = (int)((x >> 17) & 3);
            }
            last = ch;
            F.push_back((uint8_t)c);
        }
    }
    const uint64_t l_pac = F.size();
    if (l_pac == 0) return GALN_EINVAL;
    std::vector<uint8_t> pac((l_pac + 3) / 4, 0);
    for (uint64_t i = 0; i < l_pac; ++i) pac[i >> 2] |= (uint8_t)(F[i] << ((~i & 3) << 1));
    if (l_pac % 4 == 0) pac.push_back(0);
    pac.push_back((uint8_t)(l_pac % 4));
    rc = write_bytes(prefix + ".pac", pac.data(), pac.size());
    if (rc) return rc;
    std::string ann, amb;
    char line[256];
    snprintf(line, sizeof line, "%llu %d %u\n", (unsigned long long)l_pac, (int)recs.size(), 11u);
    ann += line;
    for (size_t i = 0; i < recs.size(); ++i) {
        ann += "0 " + recs[i].name + " " + recs[i].anno + "\n";
        snprintf(line, sizeof line, "%lld %d %d\n", (long long)rec_off[i], (int)rec_len[i], rec_ambs[i]);
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

int build_text(const uint8_t *fwd, uint64_t l_pac, const std::string &prefix, galn_build_stats *stats, double ms_before)
{
    for (uint64_t i = 0; i < l_pac; ++i)
        if (fwd[i] > 3) return GALN_EINVAL;
    std::vector<uint32_t> bwt;
    std::vector<uint64_t> samples;
    uint64_t L2[5] = {0, 0, 0, 0, 0}, primary = 0;
    galn_build_stats st{};
    int rc = galn::dev_build_bwt_sa(fwd, l_pac, bwt, L2, primary, samples, &st);
    if (rc) return rc;
    const double t0 = now_ms();
    rc = write_bwt_sa(prefix, primary, L2, bwt, 2 * l_pac, samples);
    st.ms_files = ms_before + (now_ms() - t0);
    if (stats) *stats = st;
    return rc;
}

}  // namespace

extern "C" int galn_index_build_text(const uint8_t *fwd, uint64_t l_pac, const char *prefix, galn_build_stats *stats)
{
    if (!fwd || !prefix || l_pac == 0) return GALN_EINVAL;
    return build_text(fwd, l_pac, prefix, stats, 0.0);
}

extern "C" int galn_fasta_to_pac(const char *fasta, const char *prefix, uint64_t *l_pac)
{
    if (!fasta || !prefix) return GALN_EINVAL;
    std::vector<uint8_t> F;
    const int rc = fasta_to_pac(fasta, prefix, F);
    if (!rc && l_pac) *l_pac = F.size();
    return rc;
}

extern "C" int galn_index_build_fasta(const char *fasta, const char *prefix, galn_build_stats *stats)
{
    if (!fasta || !prefix) return GALN_EINVAL;
    const double t0 = now_ms();
    std::vector<uint8_t> F;
    int rc = fasta_to_pac(fasta, prefix, F);
    if (rc) return rc;
    return build_text(F.data(), F.size(), prefix, stats, now_ms() - t0);
}
