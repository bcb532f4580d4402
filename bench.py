#!/usr/bin/env python
"""Throughput of the `bwa aln` search on one or more B200s: reads/s on the aDNA workload.

Workload (the reference's aDNA-batched configuration, synthetic and seeded): a 100 Mbp reference at 45% GC
in 10 contigs with 5% interspersed 300 bp repeat families (copies at 10% divergence), indexed in BWA format;
2,000,000 single-end reads per GPU with log-normal lengths (mean 50, 25-120 bp), 0.5% substitutions, 5' C->T
and 3' G->A deamination (30% at the end, x0.5 per base), 3% random reads; options -l 1024 -n 0.01 -o 2.

One step = one galn_aln_run_batch call (the public C ABI) over all reads of the GPU: reads from pinned host
memory, H2D, query encoding, every search tier, D2H of n_aln/records/pops/traces and assembly of the result
table. The L2 cache is flushed (a 512 MB write) before each step, outside the timed region.

  value   reads / device span (first to last search kernel, CUDA events on the library's stream): inputs
          already in HBM
  e2e     reads / wall time of the whole call (H2D + device + D2H + result assembly)
  roofline  the dominant kernel (the tier with the most device time): 32 B x the algorithmic block fetches
          of the reads it finished / its time; also against the device's random 32-B gather peak, swept over
          buffer sizes and loads in flight
  cpu_baseline  the reference's own `galn aln --cpu-only` on all reads of the same workload, all host cores;
          its .sai is compared byte for byte (md5) with this build's (sai_md5_vs_reference)
  divergent  the high-divergence configuration (the same reference, 100 bp reads at 4% substitutions +
          0.5% indels, -n 6 -o 2 -e 6 -k 3 -N) at a stated fraction of its 1 M reads: persistent and plain
          engines, and the reference's .sai on a prefix
  serving  continuous batching of Poisson-arriving requests on the resident index, p50/p99 latency, every
          request's .sai against the plain launch and against the reference's own run of that request

--impl reference times only the reference's CPU path (rank 0; other ranks exit at once).
--index-build times `galn index` instead (the GPU index builder on the workload's reference; see index_bench).
--profile-case warp_steady runs the fixed warp-tier case that ncu captures (see profile_warp_steady).
"""
from __future__ import annotations

import argparse
import datetime
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "reads/s, .sai md5-identical (served vs plain launch, same B200); p50/p99 latency"
TIER_NAMES = {0: "search tier 0 (thread per read, persistent claim, CUDA graph)",
              1: "warp tier (one warp per heavy read, entries of a score bucket spread over lanes)",
              2: "thread tiers (free-list stacks up to the max_entries cut-off)"}
FUSED_NAME = ("fused_kernel: the first tier (thread per read) and the warp tier in one persistent launch, "
              "heavy reads handed over through a device queue, CUDA graph")
WORKLOAD_DESC = {
    "adna": "aDNA batched: 100 Mbp reference (45% GC, 10 contigs, 5% repeats), 2,000,000 reads per GPU, "
            "log-normal 25-120 bp, deaminated, 3% random; -l 1024 -n 0.01 -o 2",
    "plain_small": "plain aln: 1 Mbp uniform reference, 20,000 x 100 bp reads per GPU; default options",
    "divergent": "high divergence: 100 Mbp aDNA-like reference, 1,000,000 x 100 bp reads per GPU at 4% "
                 "substitutions + 0.5% indels; -n 6 -o 2 -e 6 -k 3 -N",
    "genome": "genome scale: 3.1 Gbp repeat-rich reference in 24 contigs with N runs (text above 2^32), "
              "10,000,000 x 150 bp reads per GPU at scale 1; default options",
}
L2_NOTE = "flushed before every step (512 MB device write, outside the timed region)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# DRAM bytes per pop of the warp tier, from one ncu capture of it on a steady-state aDNA case (60,000 heavy
# reads, 534.5 M pops, every warp busy): 34.1 GB read + 31.4 GB written.
WARP_DRAM_BYTES_PER_POP = (34.1e9 + 31.4e9) / 534.5e6


# DRAM bytes per item and pass of the index builder's radix scatter, from one ncu capture of it on a 10 Mbp
# reference (2 x 10^7 items in one pass): 245.1 MB read + 192.2 MB written.
SCATTER_DRAM_BYTES_PER_ITEM = (245.1e6 + 192.2e6) / 2e7


def scaled_traffic(dom: int, workload: str, tiers_info: dict):
    """DRAM bytes of one launch of the dominant kernel, scaled from the ncu capture by the launch's pops (the
    aDNA workload's warp tier only; None otherwise), and how it was obtained."""
    try:
        if dom != 1 or workload != "adna":
            return None, None
        pops = int((tiers_info.get("warp_counters") or {}).get("pops") or 0)
        if pops <= 0:
            return None, None
        return (WARP_DRAM_BYTES_PER_POP * pops,
                "ncu dram__bytes_read.sum + dram__bytes_write.sum of the warp tier on a steady-state aDNA case "
                "(65.5 GB for 534.5 M pops), scaled by this launch's pops")
    except (TypeError, ValueError, AttributeError):
        return None, None


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload_config(args, world: int, n_reads: int, opts: list[str]) -> dict:
    """The workload as both arms name it (the same keys and values in the reference arm's line)."""
    return {"workload": WORKLOAD_DESC[args.workload], "scale": args.scale, "reads_scale": args.reads_scale,
            "reads_per_gpu": n_reads, "options": " ".join(opts), "l2": L2_NOTE,
            "parallelism": f"{world} independent GPU shards (reads split, index replicated)"}


def prepare(workload: str, scale: float, rank: int, device: int, data_dir: str | None, reads_scale=None,
            reference_builder: bool = False):
    """Reference + BWA index + this rank's reads, cached on disk. The index is built on this GPU by `galn
    index`, or by the reference's own CPU builder for the reference arm when that is built (the files are
    the same bytes)."""
    from galn_b200 import synth
    d = data_dir or os.path.join(tempfile.gettempdir(), f"galn_bench_{workload}_{scale}_r{rank}")
    os.makedirs(d, exist_ok=True)
    t = time.time()
    ref, reads, opts = synth.workload(workload, scale, seed=1, reads_scale=reads_scale)
    if rank:
        _, reads, _ = synth.workload(workload, scale, seed=1 + 7919 * rank, reads_scale=reads_scale)
    prefix = os.path.join(d, "ref")
    if not os.path.exists(prefix + ".bwt"):
        synth.write_fasta(prefix + ".fa", ref)
        ref_builder = None
        if reference_builder:
            import oracle
            ref_builder = oracle.INDEX_REF if os.path.exists(oracle.INDEX_REF) else None
        if ref_builder:
            subprocess.run([ref_builder, "-f", prefix + ".fa", prefix], check=True, capture_output=True)
        else:
            import galn_b200
            galn_b200.index_fasta(prefix + ".fa", prefix, device)
    log(f"[bench] rank {rank}: data ready in {time.time() - t:.1f} s ({len(reads)} reads, ref {ref.total} bp)")
    return d, prefix, ref, reads, opts


def clock_sampler_start(path, device):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    try:
        f = open(path, "w")
        return subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                 "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL), f
    except OSError:
        return None, None


def clock_sampler_stop(proc, f, path):
    if proc is None:
        return None
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except subprocess.TimeoutExpired:
        proc.kill()
    f.close()
    sm, mx, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
        parts = [x.strip() for x in line.split(",")]
        if len(parts) < 9:
            continue
        try:
            sm.append(float(parts[1]))
            mx = max(mx, float(parts[2]))
        except ValueError:
            continue
        for nm, v in zip(names, parts[5:9]):
            if v.lower() == "active":
                reasons.add(nm)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------------------------
# the reference's CPU path

def sample_fastq(reads, m: int, d: str, tag: str) -> str:
    """The first m reads as a FASTQ file in d (cached)."""
    from galn_b200 import synth
    fq = os.path.join(d, f"{tag}_{m}.fq")
    if not os.path.exists(fq):
        sub = synth.Reads(reads.names[:m], reads.seq[:int(reads.off[m])], reads.off[:m + 1].copy(),
                          reads.qual[:int(reads.off[m])] if reads.qual is not None else None)
        synth.write_fastq(fq + ".part", sub)
        os.replace(fq + ".part", fq)
    return fq


def reference_run(prefix: str, fq: str, opts: list[str], out_sai: str, cores: int) -> dict:
    """One `galn aln --cpu-only` run of the reference: its search seconds and the md5 of the .sai it wrote."""
    import oracle
    if not os.path.exists(oracle.GALN_REF):
        return {"error": "reference binary oracle/_ref/galn_ref not built"}
    info = oracle.run_galn_ref(prefix, fq, opts, out_sai, workers=cores)
    if info["rc"] not in (0, 4) or "search_s" not in info:
        return {"error": "reference run failed: " + info["stderr"][-200:]}
    with open(out_sai, "rb") as f:
        md5 = hashlib.md5(f.read()).hexdigest()
    return {"search_s": info["search_s"], "n_reads": info.get("n_reads"), "md5": md5}


def cpu_reference_full(prefix, reads, opts, d, cores, m):
    """The reference's CPU path on the first m reads of the workload (all of them for the aDNA workload: one
    run, a few tens of seconds): the cpu_baseline figure and the .sai the GPU arm is compared with."""
    n = min(m, len(reads))
    fq = sample_fastq(reads, n, d, "all")
    r = reference_run(prefix, fq, opts, os.path.join(d, "ref_all.sai"), cores)
    if "error" in r:
        return None, r["error"]
    what = f"all {n} reads" if n == len(reads) else f"the first {n} reads"
    cb = dict(value=n / max(r["search_s"], 1e-3), unit="reads/s", cores=cores, kind="reference",
              sample=f"{what} of the same workload, reference `galn aln --cpu-only --cpu-workers {cores}`, "
                     f"search time from its own timing line")
    r["n"] = n
    return (cb, r), None


def gpu_reference(prefix, reads, opts, d, cores, m):
    """The reference's own GPU path (`galn aln --gpu-only`, its light tier and warp engine compiled for this
    GPU) on the first m reads, in a process of its own with a time limit: reads/s from its timing line and
    the md5 of the .sai it wrote."""
    import oracle
    if not os.path.exists(oracle.GALN_REF):
        return {"error": "reference binary oracle/_ref/galn_ref not built"}
    n = min(m, len(reads))
    fq = sample_fastq(reads, n, d, "all")
    out = os.path.join(d, "ref_gpu.sai")
    try:
        info = oracle.run_galn_ref(prefix, fq, opts, out, workers=cores, timeout=900.0, mode="--gpu-only")
    except subprocess.TimeoutExpired:
        return {"reads": n, "error": "did not finish within 900 s"}
    if info["rc"] not in (0, 4) or "search_s" not in info:
        return {"reads": n, "error": "rc %d: %s" % (info["rc"], info["stderr"][-300:])}
    with open(out, "rb") as f:
        md5 = hashlib.md5(f.read()).hexdigest()
    return {"reads": n, "reads_per_s": n / max(info["search_s"], 1e-3), "search_s": info["search_s"], "sai_md5": md5,
            "how": "reference `galn aln --gpu-only` (its GPU path; CPU workers take only what the GPU cannot), "
                   "search time from its own timing line"}


def cpu_reference_sampled(prefix, reads, opts, sample, d, steps, warmup, cores):
    """The reference arm: the reference's CPU path on a prefix of the reads grown until one run searches
    for a few seconds (its timer has 10 ms resolution), run warmup + steps times."""
    n = min(sample, len(reads))
    while True:
        fq = sample_fastq(reads, n, d, "sample")
        r = reference_run(prefix, fq, opts, os.path.join(d, "ref_sample.sai"), cores)
        if "error" in r:
            return None, r["error"]
        if r["search_s"] >= 3.0 or n >= len(reads):
            break
        n = min(len(reads), int(n * min(8.0, 4.0 / max(r["search_s"], 0.05))))
    vals = []
    for i in range(warmup + steps):
        if i > 0:
            r = reference_run(prefix, fq, opts, os.path.join(d, "ref_sample.sai"), cores)
            if "error" in r:
                return None, r["error"]
        if i >= warmup:
            vals.append(n / max(r["search_s"], 1e-3))
    return dict(value=statistics.mean(vals), unit="reads/s", cores=cores, kind="reference",
                sample=f"first {n} reads of the same workload per step, reference `galn aln --cpu-only "
                       f"--cpu-workers {cores}`, search time from its own timing line"), None


# ------------------------------------------------------------------------------------------------------------
# --index-build

def index_bench(args, rank: int, local: int) -> int:
    """--index-build: `galn index` on the workload's reference (FASTA on disk to the five bwa index files).
    value = reference bp / device span of the builder (text in HBM to results in HBM); e2e = reference
    bp / wall time of galn_index_build_fasta (FASTA parse, device build, file writes); the roofline is the
    radix scatter (24 B of keys and values read and written per item and pass); cpu_baseline = the reference's
    own CPU builder (`galn index -a cpu`, oracle/_ref/galn_index_cpu) on the same FASTA, all host threads.
    With --impl reference only the reference's builder runs. The files are compared with the reference
    builder's when it ran."""
    import filecmp
    import oracle
    from galn_b200 import synth
    if rank != 0:
        return 0
    d = args.data_dir or os.path.join(tempfile.gettempdir(), f"galn_index_{args.workload}_{args.scale}")
    os.makedirs(d, exist_ok=True)
    ref = synth.workload_reference(args.workload, args.scale, seed=1)
    fa = os.path.join(d, "ref.fa")
    if not os.path.exists(fa):
        synth.write_fasta(fa, ref)
    cores = os.cpu_count() or 1
    config = {"workload": f"bwa index of the {args.workload} reference ({ref.total} bp, {len(ref.names)} contigs)",
              "scale": args.scale}

    def run_reference():
        if not os.path.exists(oracle.INDEX_REF):
            return None
        t = time.time()
        p = subprocess.run([oracle.INDEX_REF, "-f", fa, os.path.join(d, "refix")], capture_output=True, text=True)
        return time.time() - t if p.returncode == 0 else None

    if args.impl == "reference":
        walls = []
        for i in range(args.warmup + args.steps):
            w = run_reference()
            if w is None:
                print(json.dumps({"impl": "reference", "unavailable": "reference index builder not built"}))
                return 0
            if i >= args.warmup:
                walls.append(w)
        v = ref.total / statistics.mean(walls)
        cb = dict(value=v, unit="bp/s", cores=cores, kind="reference",
                  sample=f"the whole {ref.total} bp reference, `galn index -a cpu` with {cores} threads")
        print(json.dumps({"impl": "reference", "metric": "bwa index: reference bp/s", "value": v, "unit": "bp/s",
                          "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * statistics.mean(walls), "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)", "config": config,
                          "cpu_baseline": cb, "e2e": {"value": v, "unit": "bp/s", "h2d_bytes_per_step": 0,
                                                      "d2h_bytes_per_step": 0}}))
        return 0

    import galn_b200
    from galn_b200 import build as gbuild
    gbuild.build()
    hbm, hbm_kind = peaks()
    sts, walls = [], []
    for i in range(args.warmup + args.steps):
        t = time.time()
        st = galn_b200.index_fasta(fa, os.path.join(d, "gpu"), local)
        if i >= args.warmup:
            walls.append(time.time() - t)
            sts.append(st)
    ms_dev = statistics.mean(x["ms_device"] for x in sts)
    ms_sc = statistics.mean(x["ms_scatter"] for x in sts)
    sc_bytes = 24.0 * sts[0]["scatter_items"]
    wref = run_reference()
    same = None
    if wref is not None:
        same = all(filecmp.cmp(os.path.join(d, "gpu." + e), os.path.join(d, "refix." + e), shallow=False)
                   for e in ("pac", "ann", "amb", "bwt", "sa"))
    n = sts[0]["n"]
    d2h = os.path.getsize(os.path.join(d, "gpu.bwt")) + os.path.getsize(os.path.join(d, "gpu.sa")) - 40 - 56
    line = {"metric": "bwa index: reference bp/s (five files byte-identical to the reference builder's)",
            "value": ref.total / (ms_dev / 1e3), "unit": "bp/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_dev, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)", "config": config,
            "e2e": {"value": ref.total / statistics.mean(walls), "unit": "bp/s", "h2d_bytes_per_step": ref.total,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "kernel": "radix_scatter (all passes of all doubling rounds)",
                         "achieved": sc_bytes / (ms_sc / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": sc_bytes / (ms_sc / 1e3) / 1e9 / hbm, "peak_kind": hbm_kind,
                         "traffic": SCATTER_DRAM_BYTES_PER_ITEM * sts[0]["scatter_items"],
                         "traffic_how": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one radix_scatter launch "
                                        "on a 10 Mbp reference (437.3 MB for 2 x 10^7 items), scaled by the items of "
                                        "all scatter launches of this build"},
            "builder": {"text_symbols": n, "rounds": sts[0]["rounds"], "radix_passes": sts[0]["sort_passes"],
                        "sorted_items": sts[0]["sorted_items"], "ms_scatter": ms_sc,
                        "ms_copies": statistics.mean(x["ms_copies"] for x in sts),
                        "ms_host_files": statistics.mean(x["ms_files"] for x in sts)},
            "identical_to_reference_builder": same}
    if wref is not None:
        line["cpu_baseline"] = dict(value=ref.total / wref, unit="bp/s", cores=cores, kind="reference",
                                    sample=f"the whole {ref.total} bp reference, `galn index -a cpu` with {cores} threads")
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------------------------
# sub-records of the default run

def gather_sweep(device: int, ix_bytes: int) -> dict:
    """The device's random 32-byte sector read rate over buffer sizes (from a quarter of L2 to 32x it) and
    loads in flight per thread (galn_gather_peak_ex, best of 5 launches each)."""
    import galn_b200
    spans = [32 << 20, 128 << 20, 1 << 30, 2 << 30, 4 << 30]
    table = []
    for span in spans:
        for inf in (2, 4, 8, 16):
            g = galn_b200.gather_peak(device, span, inf, 5)
            table.append({"bytes": span, "in_flight": inf, "gbs": g})
    ix_pow2 = 1 << max(20, (ix_bytes - 1).bit_length())
    best = lambda rows: max((r for r in rows if r["gbs"]), key=lambda r: r["gbs"], default=None)  # noqa: E731
    hbm = best([r for r in table if r["bytes"] >= (1 << 30)])
    l2 = best([r for r in table if r["bytes"] == (32 << 20)])
    ixr = best([{"bytes": ix_pow2, "in_flight": inf, "gbs": galn_b200.gather_peak(device, ix_pow2, inf, 5)}
                for inf in (4, 8, 16)])
    return {"table": table, "hbm_best": hbm, "l2_best": l2, "index_size_best": ixr}


def divergent_run(ix, ref, d: str, args, cores: int, prefix: str) -> dict:
    """The high-divergence configuration on the resident aDNA index: `div_reads_scale` of its 1 M reads
    with the persistent engine (autotuned for these options), the plain per-batch engine and the persistent
    engine on the first `div_plain_reads` of them, and the reference's own .sai of the first
    `div_ref_reads` against this build's."""
    import galn_b200
    from galn_b200 import synth
    t = time.time()
    n = max(1, int(synth.FULL_READS["divergent"] * args.div_reads_scale))
    reads, opts = synth.workload_reads("divergent", ref, n, seed=1)
    R = galn_b200.Reads(reads.ascii(), reads.off.copy())
    log(f"[bench] divergent: {n} reads generated in {time.time() - t:.1f} s")
    tune = ix.autotune(opts, R, max_sample=min(n, 4096))

    def timed(eng, rr, k, w):
        dev, e2e = [], []
        res = None
        for i in range(w + k):
            t1 = time.perf_counter()
            res = galn_b200.aln(ix, opts, rr, eng)
            dt = time.perf_counter() - t1
            if i >= w:
                e2e.append(dt)
                dev.append(ix.last_profile()["ms_device"] / 1e3)
        return len(rr) / statistics.mean(dev), len(rr) / statistics.mean(e2e), res

    pv, pe, pres = timed(galn_b200.GALN_ENGINE_PERSISTENT, R, 2, 1)
    m = min(n, args.div_plain_reads)
    Rm = galn_b200.Reads(R.seq[:int(R.offset[m])], R.offset[:m + 1].copy())
    sv, se, sres = timed(galn_b200.GALN_ENGINE_PERSISTENT, Rm, 1, 0)
    qv, qe, qres = timed(galn_b200.GALN_ENGINE_PLAIN, Rm, 1, 0)
    out = {"reads": n, "reads_fraction": args.div_reads_scale, "options": " ".join(opts), "autotuned": tune,
           "persistent": {"value": pv, "e2e": pe},
           "same_reads": {"reads": m, "persistent": sv, "plain": qv, "ratio": sv / qv,
                          "sai_identical": sres.sai_bytes() == qres.sai_bytes()},
           "pops_per_read": float(pres.pops.astype("float64").mean())}
    k = min(n, args.div_ref_reads)
    if k > 0 and args.cpu_sample > 0:
        fq = sample_fastq(reads, k, d, "div")
        rr = reference_run(prefix, fq, opts, os.path.join(d, "ref_div.sai"), cores)
        Rk = galn_b200.Reads(R.seq[:int(R.offset[k])], R.offset[:k + 1].copy())
        mine = hashlib.md5(galn_b200.aln(ix, opts, Rk).sai_bytes()).hexdigest()
        out["reference"] = {"reads": k, "error": rr["error"]} if "error" in rr else {
            "reads": k, "reads_per_s": k / max(rr["search_s"], 1e-3), "cores": cores,
            "sai_md5": rr["md5"], "sai_md5_vs_reference": rr["md5"] == mine}
    return out


def serving_run(ix, ref, n_requests: int, seed: int, rate_hz: float, scale: float, d: str, prefix: str,
                check_reference: bool, cores: int):
    """The serving configuration on the resident index: Poisson arrivals, requests of 1k-500k reads
    (log-uniform, times `scale`), lengths 36-150 bp, half default and half aDNA options. Returns reads/s and
    submit-to-result latency percentiles, next to the same requests as plain per-request launches in
    arrival order (one at a time), whether every request's .sai is the same both ways, and (check_reference)
    whether every request's .sai equals the reference's own run of that request."""
    import numpy as np

    import galn_b200
    from galn_b200 import synth
    t = time.time()
    reqs = synth.serving_requests(n_requests, seed, ref, scale=scale, rate_hz=rate_hz)
    items = [(r["t_arrival"], r["opts"], galn_b200.Reads(r["reads"].ascii(), r["reads"].off.copy())) for r in reqs]
    total = sum(len(x[2]) for x in items)
    log(f"[bench] serving: {len(items)} requests, {total} reads generated in {time.time() - t:.1f} s")
    srv = galn_b200.Server(ix)
    t0 = time.perf_counter()
    ids, t_sub = [], []
    for t_arr, opts, reads in items:
        dt = t_arr - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        t_sub.append(time.perf_counter() - t0)
        ids.append(srv.submit(opts, reads))
    outs = [srv.wait(i) for i in ids]
    t_end = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    service, same = [], True
    for (t_arr, opts, reads), o in zip(items, outs):
        t1 = time.perf_counter()
        p = galn_b200.aln(ix, opts, reads, galn_b200.GALN_ENGINE_PLAIN)
        service.append(time.perf_counter() - t1)
        same = same and p.sai_bytes() == o.sai_bytes()
    t_free, lat = 0.0, []
    for (t_arr, _, _), sv in zip(items, service):
        start = max(t_arr, t_free)
        t_free = start + sv
        lat.append(t_free - t_arr)
    lat = np.array(lat) * 1e3
    out = {"requests": len(items), "reads": total, "arrival_rate_hz": rate_hz,
           "reads_per_s": total / max(t_end - t_sub[0], 1e-9), "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
           "steps": st["steps"], "device_busy_s": st["busy_ms"] / 1e3,
           "plain_per_request": {"reads_per_s": total / sum(service), "p50_ms": float(np.percentile(lat, 50)),
                                 "p99_ms": float(np.percentile(lat, 99)),
                                 "latency": "FIFO queue of one-at-a-time launches with the same arrivals"},
           "sai_identical_served_vs_plain": bool(same)}
    if check_reference:
        t = time.time()
        ok, checked, errs = True, 0, []
        for i, (req, o) in enumerate(zip(reqs, outs)):
            fq = os.path.join(d, f"serve_req{i}.fq")
            if not os.path.exists(fq):
                synth.write_fastq(fq + ".part", req["reads"])
                os.replace(fq + ".part", fq)
            rr = reference_run(prefix, fq, req["opts"], os.path.join(d, f"serve_req{i}.sai"), cores)
            if "error" in rr:
                errs.append(rr["error"])
                continue
            checked += 1
            ok = ok and rr["md5"] == hashlib.md5(o.sai_bytes()).hexdigest()
        out["sai_md5_vs_reference"] = {"requests_checked": checked, "all_identical": bool(ok and checked == len(reqs)),
                                       "errors": errs[:3], "seconds": round(time.time() - t, 1)}
    return out


def profile_warp_steady(args, local: int) -> int:
    """--profile-case warp_steady: the warp tier in its steady state, for ncu captures. From the aDNA workload
    (100 Mbp reference, 2,000,000 reads, -l 1024 -n 0.01 -o 2) it takes the first 60,000 reads that the first
    tier hands to the warp tier and that need 2,000-50,000 pops: no read long enough to run alone at the end of
    the launch, so counters describe the kernel while all warps are busy. They are searched as one bwa batch
    with -m 100000 (none of them comes near that cut-off, so their results are those of the full workload)
    and a 1024-chunk arena per warp (64 Ki entries), which keeps the device footprint near 4 GB. The search
    runs twice: the second launch of warp_kernel is the one to capture (ncu -k regex:warp_kernel -s 1 -c 1).
    Each run prints its tier times."""
    import numpy as np

    import galn_b200
    d, prefix, ref, reads, opts = prepare("adna", 1.0, 0, local, args.data_dir, None)
    full = galn_b200.Reads(reads.ascii(), reads.off.copy())
    ix = galn_b200.Index(prefix, device=local)
    ix.set_trace(False)
    sel_path = os.path.join(d, "warp_steady_reads.npy")
    if not os.path.exists(sel_path):
        ix.set_tuning(t0_cap=1024, keep_stats=True)
        r = galn_b200.aln(ix, opts, full)
        prof = ix.last_profile(len(full))
        sel = np.nonzero((prof["tier"] == 1) & (r.pops >= 2000) & (r.pops <= 50000))[0][:60000]
        np.save(sel_path, sel)
    sel = np.load(sel_path)
    sub = galn_b200.Reads.from_strings([bytes(full.seq[full.offset[i]:full.offset[i + 1]]) for i in sel])
    sub.batch = np.zeros(len(sel), np.int32)
    ix.set_tuning(t0_cap=1024, keep_stats=False)
    ix.set_warp_tier(True, 1024)
    a = list(opts) + ["-m", "100000"]
    for _ in range(2):
        r = galn_b200.aln(ix, a, sub)
        p = ix.last_profile()
        print(json.dumps(dict(case="warp_steady", reads=len(sub), ms_tier=[round(x, 3) for x in p["ms_tier"][:2]],
                              pops=int(r.pops.sum()))), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="adna", choices=sorted(WORKLOAD_DESC))
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--reads-scale", type=float, default=None, help="reads at this fraction of the workload's")
    ap.add_argument("--engine", default="persistent", choices=["persistent", "plain"])
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-engine comparison")
    ap.add_argument("--cpu-sample", type=int, default=200_000,
                    help="first reads of the reference arm's sample (0: no reference runs in the GPU arm)")
    ap.add_argument("--ref-reads", type=int, default=2_000_000,
                    help="reads of the GPU arm's reference run (its cpu_baseline and .sai md5 check)")
    ap.add_argument("--reference-gpu", action="store_true",
                    help="also time the reference's own GPU path (`galn aln --gpu-only`) on the same reads")
    ap.add_argument("--data-dir", default=None)
    ap.add_argument("--trace", action="store_true", help="compute per-read trace hashes (verification mode)")
    ap.add_argument("--t0-cap", type=int, default=1024, help="first-tier stack entries per thread")
    ap.add_argument("--warp-arena", type=int, default=8192, help="warp-tier stack chunks (64 entries) per warp")
    ap.add_argument("--serve-requests", type=int, default=40, help="requests in the serving run (0: none)")
    ap.add_argument("--no-serve-reference", dest="serve_reference", action="store_false",
                    help="skip the reference runs of the served requests")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false")
    ap.add_argument("--autotune-sample", type=int, default=2_000_000,
                    help="reads the autotuner times (the whole aDNA workload: a smaller sample holds fewer of the "
                         "heaviest reads and picked launch forms that were slower on all reads)")
    ap.add_argument("--serve-rate", type=float, default=16.0, help="request arrival rate (per second)")
    ap.add_argument("--div-reads-scale", type=float, default=0.1,
                    help="fraction of the high-divergence configuration's 1 M reads (0: skip it)")
    ap.add_argument("--div-plain-reads", type=int, default=20_000,
                    help="high-divergence reads timed with both engines")
    ap.add_argument("--div-ref-reads", type=int, default=3_000,
                    help="high-divergence reads compared with the reference's .sai")
    ap.add_argument("--no-gather-sweep", dest="gather_sweep", action="store_false")
    ap.add_argument("--index-build", action="store_true", help="time `galn index` on the workload's reference")
    ap.add_argument("--profile-case", choices=["warp_steady", "gather", "t0_small"], default=None)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cores = os.cpu_count() or 1

    if args.index_build:
        return index_bench(args, rank, local)
    if args.profile_case == "gather":
        # the random 32-byte gather probe alone, for a capture of its DRAM sectors: a 1 GiB buffer, 8 sectors in
        # flight per thread, one warm-up and two timed launches
        import galn_b200
        from galn_b200 import build as gbuild
        gbuild.build()
        print(json.dumps({"case": "gather", "bytes": 1 << 30, "in_flight": 8,
                          "gbs": galn_b200.gather_peak(local, 1 << 30, 8, 2)}))
        return 0
    if args.profile_case == "t0_small":
        # the first tier on one bwa batch of the aDNA workload (its first 262,144 reads), two launches of the
        # two-launch form; capture the first search_kernel launch (ncu -k regex:search_kernel -c 1)
        import galn_b200
        d, prefix, ref, reads, opts = prepare("adna", 1.0, 0, local, args.data_dir, None)
        m = 262144
        R = galn_b200.Reads(reads.ascii()[:int(reads.off[m])], reads.off[:m + 1].copy())
        ix = galn_b200.Index(prefix, device=local)
        ix.set_trace(False)
        ix.set_tuning(t0_cap=256, t0_block=256)
        for _ in range(2):
            galn_b200.aln(ix, opts, R)
            p = ix.last_profile()
            print(json.dumps(dict(case="t0_small", reads=m, ms_tier=[round(x, 3) for x in p["ms_tier"][:2]])))
        return 0
    if args.profile_case:
        return profile_warp_steady(args, local)
    if args.impl == "reference":
        if rank != 0:
            return 0
        d, prefix, ref, reads, opts = prepare(args.workload, args.scale, 0, local, args.data_dir, args.reads_scale,
                                              reference_builder=True)
        cb, why = cpu_reference_sampled(prefix, reads, opts, args.cpu_sample, d, args.steps, args.warmup, cores)
        if cb is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return 0
        n = len(reads)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "reads/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * n / cb["value"],
                "ms_per_step_how": f"the {n} reads of one step of the GPU arm at the sample's rate",
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                "data": "synthetic: seeded reference and reads with the workload's shapes (no public dataset here)",
                "config": workload_config(args, args.gpus, n, opts),
                "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "reads/s", "h2d_bytes_per_step": 0,
                                            "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import numpy as np
    import torch
    import torch.distributed as dist

    import galn_b200
    from galn_b200 import build as gbuild
    gbuild.build()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    d, prefix, ref, reads, opts = prepare(args.workload, args.scale, rank, local, args.data_dir, args.reads_scale)
    n = len(reads)
    # pinned host inputs
    seq_h = torch.empty(len(reads.seq), dtype=torch.uint8, pin_memory=True)
    seq_h.numpy()[:] = reads.ascii()
    off_h = torch.empty(n + 1, dtype=torch.int64, pin_memory=True)
    off_h.numpy()[:] = reads.off
    R = galn_b200.Reads(seq_h.numpy(), off_h.numpy())
    ix = galn_b200.Index(prefix, device=local)
    ix.set_trace(args.trace)
    ix.set_tuning(t0_cap=args.t0_cap)
    ix.set_warp_tier(True, args.warp_arena)
    engine = galn_b200.GALN_ENGINE_PERSISTENT if args.engine == "persistent" else galn_b200.GALN_ENGINE_PLAIN
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def barrier():
        if world > 1:
            dist.barrier()

    tier_ms_steps = []

    def run_steps(eng, k, w, keep_tiers=False):
        md5 = set()
        e2e, dev, tier0, launches = [], [], [], 0
        res = None
        for i in range(w + k):
            flush.fill_(i & 255)
            torch.cuda.synchronize()
            t = time.perf_counter()
            res = galn_b200.aln(ix, opts, R, eng)
            dt = time.perf_counter() - t
            prof = ix.last_profile()
            st = ix.last_stats()
            if i >= w:
                e2e.append(dt)
                dev.append(prof["ms_device"] / 1e3)
                tier0.append(prof["ms_tier"][0] / 1e3)
                if keep_tiers:
                    tier_ms_steps.append(list(prof["ms_tier"]))
                launches += st["launches"]
                md5.add(hashlib.md5(res.sai_bytes()).hexdigest())
        return e2e, dev, tier0, launches, md5, res

    # the autotuner picks the thread/warp split for these options on a sample (untimed), then warm-up
    tune = None
    if args.autotune and engine == galn_b200.GALN_ENGINE_PERSISTENT:
        tune = ix.autotune(opts, R, max_sample=args.autotune_sample)
        log(f"[bench] autotuner: {tune}")
    for _ in range(args.warmup):
        galn_b200.aln(ix, opts, R, engine)
    barrier()
    torch.cuda.synchronize()
    cpath = os.path.join(d, f"clocks_{rank}.csv")
    proc, cf = clock_sampler_start(cpath, local)
    e2e, dev, tier0, launches, md5, res = run_steps(engine, args.steps, 0, keep_tiers=True)
    torch.cuda.synchronize()
    barrier()
    clocks = clock_sampler_stop(proc, cf, cpath)

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    e2e_s = max_over_ranks(statistics.mean(e2e))
    dev_s = max_over_ranks(statistics.mean(dev))
    total_reads = n * world

    # roofline of the dominant kernel: algorithmic block fetches of the reads the first tier finished
    if tune:
        ix.set_tuning(t0_cap=tune["t0_cap"], t0_block=tune["block"], keep_stats=True)
    else:
        ix.set_tuning(t0_cap=args.t0_cap, keep_stats=True)
    galn_b200.aln(ix, opts, R, engine)
    prof = ix.last_profile(n)
    tiers_info = {"ms": [round(x, 3) for x in prof["ms_tier"]], "reads": prof["tier_reads"],
                  "threads": prof["tier_threads"],
                  "fetches_finished": [int(prof["fetch"][prof["tier"] == t].astype(np.int64).sum()) for t in range(8)]}
    tiers_info["warp_counters"] = ix.warp_counters()
    tiers_info["warp_queue"] = ix.last_warp_queue()
    fetch_all = int(prof["fetch"].astype(np.int64).sum())
    ix.set_tuning(t0_cap=args.t0_cap, keep_stats=False)
    peak, peak_kind = peaks()
    # the dominant kernel: the tier with the most device time per step (timed steps); its algorithmic bytes
    # are 32 B x the block fetches of the reads it finished
    tier_ms = [statistics.mean(col) for col in zip(*tier_ms_steps)]
    dom = max(range(len(tier_ms)), key=lambda t: tier_ms[t])
    dom_s = tier_ms[dom] / 1e3
    fetch_dom = tiers_info["fetches_finished"][dom]
    tiers_info["fused"] = bool(prof.get("fused"))
    if tiers_info["fused"] and dom == 0:
        # one launch ran both the first tier and the warp tier: its work is every read either finished
        fetch_dom += tiers_info["fetches_finished"][1]
    achieved = 32.0 * fetch_dom / dom_s / 1e9
    ix_bytes = os.path.getsize(prefix + ".bwt")   # the occ64 index has the .bwt body's size
    sweep = gather_sweep(local, ix_bytes) if args.gather_sweep else None
    traffic, traffic_how = scaled_traffic(dom, args.workload, tiers_info)

    plain = None
    if not args.no_plain and engine != galn_b200.GALN_ENGINE_PLAIN:
        pe2e, pdev, _, _, pmd5, _ = run_steps(galn_b200.GALN_ENGINE_PLAIN, min(3, max(1, args.steps // 2)), 1)
        plain = {"value": total_reads / max_over_ranks(statistics.mean(pdev)),
                 "e2e": total_reads / max_over_ranks(statistics.mean(pe2e)), "sai_md5_same": pmd5 == md5}

    divergent = None
    if args.workload == "adna" and args.div_reads_scale > 0 and rank == 0 and world == 1:
        divergent = divergent_run(ix, ref, d, args, cores, prefix)

    serving = None
    if args.serve_requests > 0 and args.workload == "adna":
        serving = serving_run(ix, ref, args.serve_requests, 1000 + rank, args.serve_rate, args.scale, d, prefix,
                              args.serve_reference and args.cpu_sample > 0 and world == 1, cores)

    cpu, ref_full = None, None
    if rank == 0 and world == 1 and args.cpu_sample > 0:
        got, why = cpu_reference_full(prefix, reads, opts, d, cores, args.ref_reads)
        if got is None:
            log("[bench] cpu baseline unavailable:", why)
        else:
            cpu, ref_full = got
            if ref_full["n"] < n:   # this build's .sai of the same prefix
                k = ref_full["n"]
                Rk = galn_b200.Reads(R.seq[:int(R.offset[k])], R.offset[:k + 1].copy())
                ref_full["gpu_md5"] = hashlib.md5(galn_b200.aln(ix, opts, Rk, engine).sai_bytes()).hexdigest()
    ref_gpu = None
    if args.reference_gpu and rank == 0 and world == 1:
        ref_gpu = gpu_reference(prefix, reads, opts, d, cores, args.ref_reads)
        if "sai_md5" in ref_gpu:
            mine = (ref_full or {}).get("gpu_md5") if ref_gpu["reads"] < n else (sorted(md5)[0] if len(md5) == 1 else None)
            ref_gpu["sai_md5_vs_this_build"] = ref_gpu["sai_md5"] == mine
            if ref_full and ref_full["n"] == ref_gpu["reads"]:
                ref_gpu["sai_md5_vs_reference_cpu"] = ref_gpu["sai_md5"] == ref_full["md5"]
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    h2d = int(len(reads.seq) + 8 * (n + 1))
    d2h = int(4 * n + 8 * (n + 1) + 16 * n + 24 * int(res.rec_offset[-1]))
    hbm_g = sweep["hbm_best"] if sweep else None
    l2_g = sweep["l2_best"] if sweep else None
    ix_g = sweep["index_size_best"] if sweep else None
    frac_of = lambda g: achieved / g["gbs"] if g and g.get("gbs") else None  # noqa: E731
    line = {
        "metric": METRIC, "value": total_reads / dev_s, "unit": "reads/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * e2e_s, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64",
        "data": "synthetic: seeded reference and reads with the workload's shapes (no public dataset here)",
        "config": workload_config(args, world, n, opts),
        "search": {"engine": args.engine, "trace_hashes": bool(args.trace), "autotuned": tune},
        "e2e": {"value": total_reads / e2e_s, "unit": "reads/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_how": traffic_how, "peak_kind": peak_kind,
                     "kernel": FUSED_NAME if tiers_info["fused"] and dom == 0 else TIER_NAMES[min(dom, 2)],
                     "algorithmic_bytes_per_launch": 32 * fetch_dom, "fetches_all_tiers": fetch_all,
                     "ms_per_launch": 1e3 * dom_s,
                     "gather_peak_gbs": hbm_g["gbs"] if hbm_g else None,
                     "frac_of_gather_peak": frac_of(hbm_g),
                     "gather_l2_peak_gbs": l2_g["gbs"] if l2_g else None,
                     "frac_of_gather_l2_peak": frac_of(l2_g),
                     "gather_index_size_peak_gbs": ix_g["gbs"] if ix_g else None,
                     "frac_of_gather_index_size_peak": frac_of(ix_g),
                     "gather_peak_how": "galn_gather_peak_ex: random 32-B sectors, best over buffers of 1-4 GiB "
                                        "(HBM), of 32 MiB (L2) and of the index's size (next power of two), each "
                                        "over 2-16 sectors in flight per thread, best of 5 launches",
                     "gather_sweep": sweep["table"] if sweep else None},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "sai_md5": sorted(md5),
        "deterministic": len(md5) == 1,
        "ms_device_per_step": 1e3 * dev_s,
        "tiers": tiers_info,
    }
    if ref_full:
        line["sai_md5_reference"] = ref_full["md5"]
        if "gpu_md5" in ref_full:
            line["sai_md5_vs_reference"] = ref_full["md5"] == ref_full["gpu_md5"]
        else:
            line["sai_md5_vs_reference"] = len(md5) == 1 and ref_full["md5"] in md5
        line["sai_md5_vs_reference_reads"] = ref_full["n"]
    if ref_gpu:
        line["reference_gpu"] = ref_gpu
    if plain:
        line["plain_engine"] = plain
    if divergent:
        line["divergent"] = divergent
    if serving:
        line["serving"] = serving
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
