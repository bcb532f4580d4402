"""Regenerates the golden fixtures under tests/golden/ from the reference itself.

Needs the reference sources (the oracle Makefile builds oracle/_ref/galn_ref and galn_index_cpu from
them); run once in a checkout where they are present:

    python tests/golden/make_golden.py

For each case it writes the inputs (reference FASTA, index files from the reference's own builder,
reads), the .sai written by the reference's `galn aln --cpu-only -dt 1`, and a per-read table
(n_aln, n_pops, trace hash, peak stack size) from the reference's aln_search_host. Synthetic inputs come
from galn_b200.synth with fixed seeds.
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from galn_b200 import synth  # noqa: E402


def edge_reads_fastq(path: str) -> None:
    """Hand-built records for the reader's and the search's edge cases: ambiguous bases, '-', lower case,
    CRLF line ends, multi-line FASTA records, an empty read, a malformed record in the middle (it ends a
    batch), very short and very long reads, a read of all N."""
    rng = np.random.Generator(np.random.PCG64(77))
    ref = open(os.path.join(HERE, "small", "ref.fa")).read().split("\n", 1)[1].replace("\n", "")
    def frag(L, pos=None):
        p = int(rng.integers(0, len(ref) - L)) if pos is None else pos
        return ref[p:p + L]
    recs = []
    def fq(name, s, crlf=False):
        nl = "\r\n" if crlf else "\n"
        recs.append(f"@{name} comment here{nl}{s}{nl}+{nl}{'I' * len(s)}{nl}")
    fq("plain100", frag(100))
    fq("withN", frag(40) + "NN" + frag(30))
    fq("dash", frag(50)[:20] + "-" + frag(50)[21:])
    fq("lower", frag(80).lower())
    fq("crlf", frag(60), crlf=True)
    fq("allN", "N" * 50)
    fq("short1", "A")
    fq("short5", frag(5))
    fq("short12", frag(12))
    recs.append("@empty\n\n+\n\n")
    fq("long300", frag(300))
    fq("long1000", frag(1000))
    s = frag(120)
    fq("mismatch", s[:30] + ("A" if s[30] != "A" else "C") + s[31:90] + ("G" if s[90] != "G" else "T") + s[91:])
    fq("ins", frag(70)[:35] + "ACG" + frag(70)[35:])
    recs.append("@malformed\n" + frag(40) + "\n+\n" + "I" * 10 + "\n")
    fq("after_malformed", frag(90))
    recs.append(">fasta_rec desc\n" + frag(45) + "\n" + frag(45) + "\n")
    fq("multiline_q", frag(64))
    for i in range(40):
        L = int(rng.integers(20, 140))
        t = list(frag(L))
        for _ in range(int(rng.integers(0, 4))):
            j = int(rng.integers(0, L))
            t[j] = "ACGT"[int(rng.integers(0, 4))]
        fq(f"rnd{i}", "".join(t))
    with open(path, "w") as f:
        f.write("".join(recs))


CASES = [
    # name, reference dir, reads spec, options
    ("plain", "small", dict(kind="plain_small", n=2000, seed=11), []),
    ("adna", "small", dict(kind="adna", n=3000, seed=12), synth.ADNA_OPTS),
    ("divergent", "small", dict(kind="divergent", n=60, seed=13), synth.DIVERGENT_OPTS),
    ("genome", "genome", dict(kind="genome", n=1500, seed=14), []),
    ("edge_default", "small", dict(kind="edge"), []),
    ("edge_loggap", "small", dict(kind="edge"), ["-L", "-n", "3", "-e", "2", "-R", "5", "-dt", "16"]),
    ("edge_seed", "small", dict(kind="edge"), ["-l", "20", "-k", "1", "-o", "2", "-d", "5", "-i", "3",
                                                "-M", "4", "-O", "9", "-E", "2"]),
    ("edge_nonstop", "small", dict(kind="edge"), ["-N", "-n", "2", "-m", "500"]),
    ("tiny_queue", "small", dict(kind="plain_small", n=500, seed=15), ["-m", "40"]),
]


def make_reads(spec, ref_obj, path):
    if spec["kind"] == "edge":
        edge_reads_fastq(path)
        return
    kind, n, seed = spec["kind"], spec["n"], spec["seed"]
    if kind == "plain_small":
        r = synth.simulate_reads(ref_obj, n, seed, 100, sub_rate=0.01, indel_rate=0.001, random_frac=0.02, prefix="p")
    elif kind == "adna":
        r = synth.simulate_reads(ref_obj, n, seed, synth.adna_lengths, sub_rate=0.005, random_frac=0.03,
                                 deaminate=0.3, prefix="a")
    elif kind == "divergent":
        r = synth.simulate_reads(ref_obj, n, seed, 100, sub_rate=0.04, indel_rate=0.005, prefix="d")
    elif kind == "genome":
        r = synth.simulate_reads(ref_obj, n, seed, 150, sub_rate=lambda x: 0.001 + 0.014 * x,
                                 indel_rate=0.0005, prefix="g")
    synth.write_fastq(path, r)


def main():
    oracle.build(ref=True)
    refs = {
        "small": synth.reference_adna(100_000, 3, n_contigs=2),
        "genome": synth.reference_genome(120_000, 4, n_contigs=3),
    }
    for name, ref in refs.items():
        d = os.path.join(HERE, name)
        os.makedirs(d, exist_ok=True)
        synth.write_fasta(os.path.join(d, "ref.fa"), ref)
        subprocess.run([oracle.INDEX_REF, "-f", os.path.join(d, "ref.fa"), os.path.join(d, "ref")], check=True,
                       capture_output=True)
    manifest = {}
    for name, refdir, spec, opts in CASES:
        d = os.path.join(HERE, "cases", name)
        os.makedirs(d, exist_ok=True)
        fq = os.path.join(d, "reads.fq")
        make_reads(spec, refs.get(refdir), fq)
        prefix = os.path.join(HERE, refdir, "ref")
        sai = os.path.join(d, "expected.sai")
        info = oracle.run_galn_ref(prefix, fq, opts, sai, workers=2)
        assert info["rc"] in (0, 4), info["stderr"]
        ob = oracle.opt_bytes(oracle.parse_aln_args(opts))
        assert open(sai, "rb").read()[4:68] == ob, "option block differs from the reference's"
        dump = oracle.ref_dump(prefix + ".bwt", fq, ob, os.path.join(d, "dump.bin"), 2)
        os.remove(os.path.join(d, "dump.bin"))
        np.savez_compressed(os.path.join(d, "per_read.npz"), n_aln=dump["n_aln"], pops=dump["pops"],
                            trace=dump["trace"], peak=dump["peak"], batch=dump["batch"], len=dump["len"])
        with open(fq, "rb") as f, gzip.open(fq + ".gz", "wb", compresslevel=9) as g:
            shutil.copyfileobj(f, g)
        os.remove(fq)
        manifest[name] = dict(ref=refdir, opts=opts, rc=info["rc"], n_reads=int(len(dump["n_aln"])),
                              sai_md5=hashlib.md5(open(sai, "rb").read()).hexdigest())
        print(name, manifest[name])
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
