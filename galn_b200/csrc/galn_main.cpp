// galn_main.cpp -- the `galn aln` and `galn index` command lines on top of the C ABI (the reference's
// galn_aln, src/galn.cu:436-1288, its usage text, src/galn.cu:144-180, and galn index,
// src/index/galn_index.c:36-71).
//
//   galn aln [options] <prefix> <reads.fq[.gz]> [> out.sai]
//   galn index [-a auto|gpu|gpu-lowmem] [-p prefix] [-t threads] [-v] [--device N] <in.fasta[.gz]>
//
// galn index writes the five files of bwa index 0.7.19; every builder choice runs the GPU builder (-a cpu
// is refused: there is no CPU path), -t is accepted and ignored, bwa's -a is/bwtsw/rb2 mean auto.
//
// Every bwa aln option keeps its meaning and default; -dt only sets the thread count written into the .sai
// header. Per-read trace hashes (the reference's --verify data) are computed only with --verify. Flags of the reference that pick CPU/GPU work sharing (--cpu-workers, --gpu-only, --cpu-interleave,
// --handoff, --handoff-when, --light-cap, --warps, --pool-gb, --alloc) are accepted and ignored: all reads run
// on the GPU. --cpu-only is refused (there is no CPU search). --device and --gpus pick the GPUs. With the
// persistent engine (the default) parsing, searching and writing overlap: bwa batches are read one at a time
// and each GPU searches what has been read so far in one call; with --engine plain the whole input is read
// first and split over the GPUs in contiguous shards whose batches keep the options of the whole input.
// Exit codes follow the reference: 1 usage/option, 2 index, 3 reads, 4 a read could not be searched,
// 5 write error, 10 CUDA error or no device (src/galn.cu:551-552, 1256-1263, 453-454, 80-83).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/galn_aln.h"

static int usage()
{
    fprintf(stderr,
            "\nProgram: galn-b200 (bwa aln search on NVIDIA B200, sm_100a)\n\n"
            "Usage:   galn aln [options] <prefix> <in.fq[.gz]>\n"
            "         galn index [-a auto|gpu|gpu-lowmem] [-p prefix] [-v] [--device N] <in.fasta[.gz]>\n\n"
            "bwa aln options (same meaning and defaults as BWA 0.7.19):\n"
            "         -n NUM    max #diff (int) or missing prob under 0.02 err rate (float) [0.04]\n"
            "         -o INT    maximum number of gap opens [1]\n"
            "         -e INT    maximum number of gap extensions, -1 for disabling long gaps [-1]\n"
            "         -i INT    do not put an indel within INT bp towards the ends [5]\n"
            "         -d INT    maximum occurrences for extending a long deletion [10]\n"
            "         -l INT    seed length [32]\n"
            "         -k INT    maximum differences in the seed [2]\n"
            "         -m INT    maximum entries in the queue [2000000]\n"
            "         -dt INT   thread count written to the .sai header, as bwa aln -t [1]\n"
            "         -M INT    mismatch penalty [3]\n"
            "         -O INT    gap open penalty [11]\n"
            "         -E INT    gap extension penalty [4]\n"
            "         -R INT    stop searching when there are >INT equally best hits [30]\n"
            "         -L        log-scaled gap penalty for long deletions\n"
            "         -N        non-iterative mode: search for all n-difference hits (slooow)\n"
            "         -f FILE   file to write output to instead of stdout\n"
            "         (not supported: -q, -b/-0/-1/-2, -I, -Y, -B)\n\n"
            "GPU options:\n"
            "         --device LIST  CUDA device(s), e.g. 0 or 0,1 [all visible]\n"
            "         --gpus INT     use the first INT visible devices [all]\n"
            "         --engine STR   persistent (default) or plain\n"
            "         -v             timing statistics on stderr\n\n");
    return 1;
}

// the pipelined CLI: reads parsed ahead of the GPUs, and the most reads one search call takes
static const int64_t kQueueReads = 4 << 20;
static const int64_t kCallReads = 4 << 20;

static double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// The whole input read first, then searched in one call per GPU (contiguous shards) and written: the form
// the plain engine is compared in.
static int run_whole(const galn_opts &opt, const char *const pos[2], const char *outfn, const std::vector<int> &devs,
                     int engine, int verbose, int verify)
{
    double t0 = now_s();
    galn_read_set rs;
    int rr = 0;
    std::thread reader([&] { rr = galn_fastq_read(pos[1], &rs); });
    std::vector<galn_index *> ix(devs.size(), nullptr);
    int ierr = 0;
    for (size_t g = 0; g < devs.size(); ++g) {
        int e = 0;
        ix[g] = galn_index_open(pos[0], devs[g], &e);
        if (!ix[g]) ierr = e;
        else galn_index_set_trace(ix[g], verify);   // per-read trace hashes only for --verify
    }
    reader.join();
    if (ierr) {
        fprintf(stderr, "[galn] cannot load the index %s.bwt (%d)\n", pos[0], ierr);
        return ierr == GALN_ECUDA ? 10 : 2;
    }
    if (rr) { fprintf(stderr, "[galn] cannot read %s\n", pos[1]); return 3; }
    double t_loaded = now_s();

    // shards: contiguous ranges; every shard carries the whole input's longest read per batch
    const galn_reads &all = rs.reads;
    int n = all.n_reads;
    int nb = 0;
    for (int r = 0; r < n; ++r) nb = std::max(nb, all.batch[r] + 1);
    std::vector<int32_t> bmax((size_t)std::max(nb, 1), 0);
    for (int r = 0; r < n; ++r)
        bmax[all.batch[r]] = std::max(bmax[all.batch[r]], (int32_t)(all.offset[r + 1] - all.offset[r]));
    size_t G = devs.size();
    std::vector<galn_results> res(G);
    std::vector<int> rc(G, 0);
    std::vector<int> s0(G + 1);
    for (size_t g = 0; g <= G; ++g) s0[g] = (int)((int64_t)n * (int64_t)g / (int64_t)G);
    std::vector<std::thread> th;
    for (size_t g = 0; g < G; ++g)
        th.emplace_back([&, g] {
            galn_reads sh;
            sh.n_reads = s0[g + 1] - s0[g];
            sh.seq = all.seq;
            sh.offset = all.offset + s0[g];
            sh.batch = all.batch + s0[g];
            sh.batch_max_len = bmax.data();
            sh.n_batches = nb;
            rc[g] = galn_aln_run_batch(ix[g], &opt, &sh, engine, &res[g]);
        });
    for (auto &t : th) t.join();
    for (size_t g = 0; g < G; ++g)
        if (rc[g]) { fprintf(stderr, "[galn] search failed on GPU %d (%d)\n", devs[g], rc[g]); return 10; }
    double t_search = now_s();

    // one result table in input order
    galn_results merged;
    std::vector<int32_t> m_n((size_t)std::max(n, 1));
    std::vector<int64_t> m_off((size_t)n + 1);
    std::vector<galn_aln1> m_rec;
    std::vector<uint64_t> m_pops((size_t)std::max(n, 1)), m_trace((size_t)std::max(n, 1));
    int64_t t = 0;
    for (size_t g = 0; g < G; ++g)
        for (int j = 0; j < res[g].n_reads; ++j) {
            int r = s0[g] + j;
            m_n[r] = res[g].n_aln[j];
            m_off[r] = t;
            m_pops[r] = res[g].n_pops[j];
            m_trace[r] = res[g].trace[j];
            int64_t k = res[g].rec_offset[j + 1] - res[g].rec_offset[j];
            m_rec.insert(m_rec.end(), res[g].rec + res[g].rec_offset[j], res[g].rec + res[g].rec_offset[j] + k);
            t += k;
        }
    m_off[n] = t;
    if (m_rec.empty()) m_rec.resize(1);
    merged.n_reads = n;
    merged.n_aln = m_n.data();
    merged.rec_offset = m_off.data();
    merged.rec = m_rec.data();
    merged.n_pops = m_pops.data();
    merged.trace = m_trace.data();
    merged._priv = nullptr;
    int werr = galn_sai_write(outfn, &opt, &merged);
    double t_end = now_s();
    long mapped = 0;
    for (int r = 0; r < n; ++r) mapped += m_n[r] > 0;
    for (int r = 0; r < n; ++r)
        if (m_n[r] < 0) fprintf(stderr, "[galn] read %d (%s): search error %d\n", r, rs.names[r], m_n[r]);
    fprintf(stderr, "[galn] %d reads (%ld with hits, %lld records) in %.2f s: load %.2f s, search %.2f s, write %.2f s\n",
            n, mapped, (long long)t, t_end - t0, t_loaded - t0, t_search - t_loaded, t_end - t_search);
    if (verbose) {
        for (size_t g = 0; g < G; ++g) {
            double ms_tot = 0, ms_k = 0;
            int tiers = 0;
            int64_t launches = 0, ovf[8];
            galn_last_run_stats(ix[g], &ms_tot, &ms_k, &tiers, &launches, ovf);
            double pops = 0;
            for (int j = 0; j < res[g].n_reads; ++j) pops += (double)res[g].n_pops[j];
            fprintf(stderr, "[galn] GPU %d: %d reads, %.2f ms (kernels %.2f ms, %.3e pops/s), %d tiers, %lld launches,"
                    " overflow T0 %lld T1 %lld T2 %lld\n", devs[g], res[g].n_reads, ms_tot, ms_k,
                    ms_k > 0 ? pops / (ms_k / 1e3) : 0.0, tiers, (long long)launches, (long long)ovf[0],
                    (long long)ovf[1], (long long)ovf[2]);
        }
    }
    for (size_t g = 0; g < G; ++g) { galn_results_free(&res[g]); galn_index_close(ix[g]); }
    galn_read_set_free(&rs);
    if (werr == 5) { fprintf(stderr, "[galn] error writing the .sai\n"); return 5; }
    return werr;
}

// The persistent engine, pipelined: a reader thread parses the input one bwa batch at a time into a queue;
// one search thread per GPU takes everything queued so far (at least one batch, at most kCallReads reads)
// as one galn_aln_run_batch call, each bwa batch keeping its own options (its batch id is local to the
// call, its longest read its own); a writer thread appends the calls' results to the .sai stream in input
// order. Parsing, searching and writing overlap, and the calls stay large.
static int run_pipelined(const galn_opts &opt, const char *const pos[2], const char *outfn, const std::vector<int> &devs,
                         int verbose, int verify)
{
    const double t0 = now_s();
    int e_in = 0;
    galn_fastq_stream *in = galn_fastq_open(pos[1], &e_in);
    if (!in) { fprintf(stderr, "[galn] cannot read %s\n", pos[1]); return 3; }
    const size_t G = devs.size();
    std::vector<galn_index *> ix(G, nullptr);
    int ierr = 0;
    for (size_t g = 0; g < G && !ierr; ++g) {
        int e = 0;
        ix[g] = galn_index_open(pos[0], devs[g], &e);
        if (!ix[g]) ierr = e;
        else galn_index_set_trace(ix[g], verify);   // per-read trace hashes only for --verify
    }
    auto close_all = [&] {
        for (size_t g = 0; g < G; ++g)
            if (ix[g]) galn_index_close(ix[g]);
        galn_fastq_close(in);
    };
    if (ierr) {
        fprintf(stderr, "[galn] cannot load the index %s.bwt (%d)\n", pos[0], ierr);
        close_all();
        return ierr == GALN_ECUDA ? 10 : 2;
    }
    const double t_loaded = now_s();
    int werr = 0;
    galn_sai_writer *w = galn_sai_open(outfn, &opt, &werr);
    if (!w) { fprintf(stderr, "[galn] error writing the .sai\n"); close_all(); return 5; }

    // parsed batches waiting for a GPU, and finished calls waiting for the writer (by call number)
    struct Call {
        std::vector<galn_read_set> sets;
        galn_results res;
        int rc = 0;
        long first_read = 0;
    };
    std::mutex mu;
    std::condition_variable cv;
    std::deque<galn_read_set> parsed;
    int64_t parsed_reads = 0;
    bool reader_done = false;
    int read_err = 0;
    double t_parse = 0;
    long next_call = 0, next_read = 0;
    std::map<long, Call *> done;
    std::thread reader([&] {
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return parsed_reads < kQueueReads; });
            }
            galn_read_set rs;
            const double tp = now_s();
            const int rc = galn_fastq_next(in, &rs);
            t_parse += now_s() - tp;
            if (rc) { read_err = rc; break; }
            if (rs.reads.n_reads == 0) { galn_read_set_free(&rs); break; }
            std::lock_guard<std::mutex> lk(mu);
            parsed_reads += rs.reads.n_reads;
            parsed.push_back(rs);
            cv.notify_all();
        }
        std::lock_guard<std::mutex> lk(mu);
        reader_done = true;
        cv.notify_all();
    });
    std::vector<double> t_search(G, 0);
    std::vector<std::thread> searchers;
    for (size_t g = 0; g < G; ++g)
        searchers.emplace_back([&, g] {
            std::vector<char> seq;
            std::vector<int64_t> off;
            std::vector<int32_t> batch;
            for (;;) {
                auto *c = new Call();
                long id;
                {
                    std::unique_lock<std::mutex> lk(mu);
                    cv.wait(lk, [&] { return !parsed.empty() || reader_done; });
                    if (parsed.empty()) { delete c; break; }
                    int64_t m = 0;
                    while (!parsed.empty() && (c->sets.empty() || m + parsed.front().reads.n_reads <= kCallReads)) {
                        m += parsed.front().reads.n_reads;
                        c->sets.push_back(parsed.front());
                        parsed.pop_front();
                    }
                    parsed_reads -= m;
                    id = next_call++;
                    c->first_read = next_read;
                    next_read += (long)m;
                    cv.notify_all();
                }
                // one call: the batches back to back, batch b of the call = its b-th bwa batch
                seq.clear(); off.assign(1, 0); batch.clear();
                for (size_t b = 0; b < c->sets.size(); ++b) {
                    const galn_reads &r = c->sets[b].reads;
                    const int64_t base = (int64_t)seq.size() - r.offset[0];
                    seq.insert(seq.end(), r.seq + r.offset[0], r.seq + r.offset[r.n_reads]);
                    for (int j = 0; j < r.n_reads; ++j) {
                        off.push_back(base + r.offset[j + 1]);
                        batch.push_back((int32_t)b);
                    }
                }
                galn_reads call;
                memset(&call, 0, sizeof(call));
                call.n_reads = (int32_t)batch.size();
                call.seq = seq.data();
                call.offset = off.data();
                call.batch = batch.data();
                memset(&c->res, 0, sizeof(c->res));
                const double ts = now_s();
                c->rc = galn_aln_run_batch(ix[g], &opt, &call, GALN_ENGINE_PERSISTENT, &c->res);
                t_search[g] += now_s() - ts;
                std::lock_guard<std::mutex> lk(mu);
                done[id] = c;
                cv.notify_all();
            }
        });

    // the writer: calls in order
    long n = 0, mapped = 0;
    long long n_rec = 0;
    int search_err = 0;
    for (long id = 0;; ++id) {
        Call *c = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return done.count(id) || (reader_done && parsed.empty() && next_call == id); });
            auto it = done.find(id);
            if (it == done.end()) break;
            c = it->second;
            done.erase(it);
        }
        if (c->rc) { if (!search_err) search_err = c->rc; }
        else {
            if (!search_err && galn_sai_append(w, &c->res) == 5) werr = 5;
            int j = 0;
            for (auto &rs : c->sets)
                for (int t = 0; t < rs.reads.n_reads; ++t, ++j) {
                    const int na = c->res.n_aln[j];
                    if (na > 0) { ++mapped; n_rec += na; }
                    if (na < 0) fprintf(stderr, "[galn] read %ld (%s): search error %d\n", c->first_read + j, rs.names[t], na);
                }
            n += c->res.n_reads;
            galn_results_free(&c->res);
        }
        for (auto &rs : c->sets) galn_read_set_free(&rs);
        delete c;
    }
    reader.join();
    for (auto &t : searchers) t.join();
    const int cerr = galn_sai_close(w);
    if (!werr) werr = cerr;
    const double t_end = now_s();
    if (read_err) { fprintf(stderr, "[galn] cannot read %s\n", pos[1]); close_all(); return 3; }
    if (search_err) { fprintf(stderr, "[galn] search failed (%d)\n", search_err); close_all(); return 10; }
    double ts = 0;
    for (double x : t_search) ts = std::max(ts, x);
    fprintf(stderr, "[galn] %ld reads (%ld with hits, %lld records) in %.2f s: load %.2f s, then parse, search and write "
            "overlapped %.2f s (parse %.2f s, search %.2f s)\n", n, mapped, n_rec, t_end - t0, t_loaded - t0,
            t_end - t_loaded, t_parse, ts);
    if (verbose) {
        for (size_t g = 0; g < G; ++g) {
            double ms_tot = 0, ms_k = 0;
            int tiers = 0;
            int64_t launches = 0, ovf[8];
            galn_last_run_stats(ix[g], &ms_tot, &ms_k, &tiers, &launches, ovf);
            fprintf(stderr, "[galn] GPU %d: search %.2f s; last call %.2f ms (kernels %.2f ms), %d tiers, %lld launches\n",
                    devs[g], t_search[g], ms_tot, ms_k, tiers, (long long)launches);
        }
    }
    close_all();
    if (werr == 5) { fprintf(stderr, "[galn] error writing the .sai\n"); return 5; }
    return werr;
}

static int index_usage()
{
    fprintf(stderr,
            "\nUsage:   galn index [-a STR] [-p prefix] [-v] [--device N] <in.fasta[.gz]>\n\n"
            "Options: -a STR   auto, gpu or gpu-lowmem (one GPU builder; bwa's is, bwtsw and rb2 mean auto) [auto]\n"
            "         -p STR   prefix of the index files [the FASTA file name]\n"
            "         -t INT   accepted and ignored\n"
            "         -v       the time of each step on stderr\n"
            "         --device INT  CUDA device [0]\n\n");
    return 1;
}

// galn index (src/index/galn_index.c:36-71): exit 1 usage, 2 the FASTA or the index files, 10 CUDA
static int index_main(int argc, char **argv)
{
    const char *prefix = nullptr, *fa = nullptr;
    int verbose = 0, device = 0;
    for (int i = 0; i < argc; ++i) {
        const char *a = argv[i], *v = i + 1 < argc ? argv[i + 1] : nullptr;
        if (!strcmp(a, "-p") && v) { prefix = v; ++i; }
        else if (!strcmp(a, "-t") && v) ++i;
        else if (!strcmp(a, "--device") && v) { device = atoi(v); ++i; }
        else if (!strcmp(a, "-v")) verbose = 1;
        else if (!strcmp(a, "--cpu")) { fprintf(stderr, "[galn index] there is no CPU builder in this build\n"); return 1; }
        else if (!strcmp(a, "-a") && v) {
            ++i;
            if (!strcmp(v, "cpu")) { fprintf(stderr, "[galn index] there is no CPU builder in this build\n"); return 1; }
            if (strcmp(v, "auto") && strcmp(v, "gpu") && strcmp(v, "gpu-lowmem") && strcmp(v, "is") &&
                strcmp(v, "bwtsw") && strcmp(v, "rb2")) {
                fprintf(stderr, "[galn index] unknown builder -a %s\n", v);
                return index_usage();
            }
        }
        else if (a[0] == '-') { fprintf(stderr, "[galn index] unknown option %s\n", a); return index_usage(); }
        else if (!fa) fa = a;
        else return index_usage();
    }
    if (!fa) return index_usage();
    if (!prefix) prefix = fa;
    galn_build_stats st{};
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = galn_index_build_fasta(fa, prefix, device, &st);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc) {
        fprintf(stderr, "[galn index] failed (%d) for %s\n", rc, fa);
        return rc == GALN_ECUDA ? 10 : 2;
    }
    if (verbose)
        fprintf(stderr, "[galn index] %llu symbols, %d doubling rounds, %d radix passes: device %.1f ms "
                "(scatter %.1f ms), copies %.1f ms, files %.1f ms, %.2f s in all\n", (unsigned long long)st.n,
                st.rounds, st.sort_passes, st.ms_device, st.ms_scatter, st.ms_copies, st.ms_files, secs);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 2) return usage();
    if (!strcmp(argv[1], "--version") || !strcmp(argv[1], "version")) { printf("%s\n", galn_version()); return 0; }
    if (!strcmp(argv[1], "index")) return index_main(argc - 2, argv + 2);
    if (strcmp(argv[1], "aln")) {
        fprintf(stderr, "[galn] unknown command '%s' (this build provides aln and index)\n", argv[1]);
        return usage();
    }
    std::vector<const char *> bwa_args;
    const char *devspec = nullptr;
    int ngpus = 0, verbose = 0, verify = 0, engine = GALN_ENGINE_PERSISTENT;
    static const char *ignored_with_value[] = {"--cpu-workers", "--cpu-interleave", "--handoff", "--handoff-when",
                                               "--light-cap", "--warps", "--pool-gb", "--alloc"};
    for (int i = 2; i < argc; ++i) {
        const char *a = argv[i];
        const char *v = i + 1 < argc ? argv[i + 1] : nullptr;
        bool skip = false;
        for (const char *ig : ignored_with_value)
            if (!strcmp(a, ig)) { if (!v) return usage(); ++i; skip = true; break; }
        if (skip) continue;
        if (!strcmp(a, "--gpu-only")) continue;
        if (!strcmp(a, "--verify")) { verify = 1; continue; }
        if (!strcmp(a, "--cpu-only")) { fprintf(stderr, "[galn] --cpu-only: this build searches on the GPU only\n"); return 1; }
        if (!strcmp(a, "-v")) { verbose = 1; continue; }
        if (!strcmp(a, "--device")) { if (!v) return usage(); devspec = v; ++i; continue; }
        if (!strcmp(a, "--gpus")) { if (!v) return usage(); ngpus = atoi(v); ++i; continue; }
        if (!strcmp(a, "--engine")) {
            if (!v) return usage();
            if (!strcmp(v, "plain")) engine = GALN_ENGINE_PLAIN;
            else if (!strcmp(v, "persistent")) engine = GALN_ENGINE_PERSISTENT;
            else return usage();
            ++i;
            continue;
        }
        bwa_args.push_back(a);
    }
    galn_opts opt;
    const char *pos[2] = {nullptr, nullptr};
    int npos = 0;
    const char *outfn = nullptr;
    char err[256] = "";
    if (galn_opts_parse((int)bwa_args.size(), bwa_args.data(), &opt, pos, 2, &npos, &outfn, err, sizeof(err)) != 0) {
        fprintf(stderr, "[galn] %s\n", err);
        return usage();
    }
    if (npos != 2) return usage();

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        fprintf(stderr, "[galn] no CUDA device found\n");
        return 10;
    }
    std::vector<int> devs;
    if (devspec) {
        for (const char *p = devspec; *p;) {
            char *e;
            long d = strtol(p, &e, 10);
            if (e == p || d < 0 || d >= ndev) { fprintf(stderr, "[galn] --device: no CUDA device '%s'\n", devspec); return 1; }
            if (std::find(devs.begin(), devs.end(), (int)d) == devs.end()) devs.push_back((int)d);
            if (*e && *e != ',') { fprintf(stderr, "[galn] --device: bad list '%s'\n", devspec); return 1; }
            p = *e == ',' ? e + 1 : e;
        }
    } else {
        int k = ngpus > 0 ? std::min(ngpus, ndev) : ndev;
        for (int d = 0; d < k; ++d) devs.push_back(d);
    }

    if (engine == GALN_ENGINE_PLAIN) return run_whole(opt, pos, outfn, devs, engine, verbose, verify);
    return run_pipelined(opt, pos, outfn, devs, verbose, verify);
}

