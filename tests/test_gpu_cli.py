"""The `galn aln` command line on the GPU: the reference's .sai bytes and exit code for every golden case with
both engines (the persistent engine's pipeline reads, searches and writes one bwa batch at a time; the plain
engine reads the whole file first), and the same bytes from both paths and from the library call on an
input of several bwa batches with a malformed record in the middle."""
import gzip
import os
import subprocess

import numpy as np
import pytest

import galn_b200
from conftest import GOLDEN, case_paths, golden_cases
from galn_b200 import build, synth

pytestmark = pytest.mark.gpu
CASES = golden_cases()


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _run(args, out):
    with open(out, "wb") as f:
        p = subprocess.run([build.CLI, "aln", *args], stdout=f, stderr=subprocess.PIPE, text=True)
    return p.returncode, p.stderr


@pytest.mark.parametrize("engine", ["persistent", "plain"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_cli_golden(name, engine, tmp_path):
    meta = CASES[name]
    p = case_paths(name, meta)
    out = str(tmp_path / "out.sai")
    rc, err = _run(["--engine", engine, *meta["opts"], os.path.join(GOLDEN, meta["ref"], "ref"), p["fq"]], out)
    assert rc == meta["rc"], err
    assert open(out, "rb").read() == open(p["sai"], "rb").read()


def test_cli_several_batches(tmp_path):
    ref = synth.reference_adna(100_000, 3, n_contigs=2)
    r = synth.simulate_reads(ref, 0x40000 + 40_000, 61, synth.adna_lengths, sub_rate=0.005, random_frac=0.03,
                             deaminate=0.3)
    prefix = os.path.join(GOLDEN, "small", "ref")
    fq = str(tmp_path / "many.fq.gz")
    a = r.ascii()
    with gzip.open(fq, "wt", compresslevel=1) as f:
        for i in range(len(r.off) - 1):
            s = a[r.off[i]:r.off[i + 1]].tobytes().decode()
            if i == 5000:   # a malformed record: it ends the first batch early
                f.write(f"@bad\n{s}\n+\n{'I' * (len(s) + 2)}\n")
            else:
                f.write(f"@r{i}\n{s}\n+\n{'I' * len(s)}\n")
    outs = {}
    for engine in ("persistent", "plain"):
        out = str(tmp_path / f"{engine}.sai")
        rc, err = _run(["--engine", engine, *synth.ADNA_OPTS, prefix, fq], out)
        assert rc in (0, 4), err
        outs[engine] = open(out, "rb").read()
    assert outs["persistent"] == outs["plain"]
    reads = galn_b200.read_fastq(fq)
    assert len(np.unique(reads.batch)) == 3
    ix = galn_b200.Index(prefix)
    assert galn_b200.aln(ix, synth.ADNA_OPTS, reads).sai_bytes() == outs["plain"]


def test_cli_output_file_option(tmp_path):
    meta = CASES["plain"]
    p = case_paths("plain", meta)
    out = str(tmp_path / "f.sai")
    rc, err = _run(["-f", out, *meta["opts"], os.path.join(GOLDEN, meta["ref"], "ref"), p["fq"]], str(tmp_path / "stdout"))
    assert rc == 0, err
    assert open(out, "rb").read() == open(p["sai"], "rb").read()
    assert os.path.getsize(str(tmp_path / "stdout")) == 0
