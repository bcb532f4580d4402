"""`galn index` on the GPU: all five files equal to the reference builder's for every golden FASTA (the
library call and the command line), the .bwt/.sa of random, repetitive and tiny texts equal to the
oracle's, a larger genome-like reference equal to the fixture builder's (pinned itself to the reference),
and an index the builder wrote searched to the reference's .sai bytes."""
import filecmp
import os
import subprocess

import numpy as np
import pytest

import galn_b200
import oracle
from conftest import GOLDEN, case_paths, golden_cases
import fixture_index as index_build
from galn_b200 import build, synth

pytestmark = pytest.mark.gpu
INDEX_CASES = sorted(os.listdir(os.path.join(GOLDEN, "index")))
EXTS = ("pac", "ann", "amb", "bwt", "sa")


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()
    oracle.build()


def _fasta(d):
    gz = os.path.join(d, "ref.fa.gz")
    return gz if os.path.exists(gz) else os.path.join(d, "ref.fa")


def _same(a, b):
    return filecmp.cmp(a, b, shallow=False)


@pytest.mark.parametrize("d", [os.path.join(GOLDEN, "index", c) for c in INDEX_CASES] +
                         [os.path.join(GOLDEN, "small"), os.path.join(GOLDEN, "genome")])
def test_golden_fasta(d, tmp_path):
    pre = str(tmp_path / "g")
    st = galn_b200.index_fasta(_fasta(d), pre)
    for ext in EXTS:
        assert _same(pre + "." + ext, os.path.join(d, "ref." + ext)), ext
    assert st["n"] == 2 * len(oracle.forward_from_pac(pre + ".pac"))
    assert st["sort_passes"] >= 8 and st["ms_device"] > 0


def test_command_line(tmp_path):
    d = os.path.join(GOLDEN, "index", "repeats")
    pre = str(tmp_path / "c")
    p = subprocess.run([build.CLI, "index", "-v", "-p", pre, _fasta(d)], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr
    for ext in EXTS:
        assert _same(pre + "." + ext, os.path.join(d, "ref." + ext)), ext
    p = subprocess.run([build.CLI, "index", "-a", "cpu", "-p", pre, _fasta(d)], capture_output=True, text=True)
    assert p.returncode == 1


def _texts():
    rng = np.random.default_rng(77)
    yield "random", rng.integers(0, 4, 250_000)
    yield "homopolymer", np.zeros(6000, np.int64)
    yield "dinucleotide", np.tile([0, 1], 4000)
    yield "period7", np.tile(rng.integers(0, 4, 7), 2000)
    u = rng.integers(0, 4, 20_000)
    yield "repeats", np.concatenate([u, rng.integers(0, 4, 100), u, 3 - u[::-1], u[:5000]])
    yield "palindrome", np.concatenate([u[:8000], 3 - u[:8000][::-1]])
    for n in (1, 2, 3, 4, 5, 15, 16, 17, 63, 64, 65, 127, 128, 129, 2047, 2048, 2049, 4095, 4096, 4097):
        yield f"len{n}", rng.integers(0, 4, n)


@pytest.mark.parametrize("name,F", list(_texts()), ids=[t[0] for t in _texts()])
def test_texts_against_oracle(name, F, tmp_path):
    F = np.asarray(F, dtype=np.uint8)
    galn_b200.index_text(F, str(tmp_path / "g"))
    oracle.index_files(F, str(tmp_path / "o"))
    for ext in ("bwt", "sa"):
        assert _same(str(tmp_path / ("g." + ext)), str(tmp_path / ("o." + ext))), ext


# suffixes the 64-bit path sorts at once, per text: small enough for several buckets and round chunks where
# the text allows it (a homopolymer's suffixes share one prefix and one group, so it needs the whole text)
WIDE_CHUNK = {"random": 31_250, "repeats": 16_000, "palindrome": 4_000}


@pytest.mark.parametrize("name,F", list(_texts()), ids=[t[0] for t in _texts()])
def test_texts_64bit_path_against_oracle(name, F, tmp_path):
    """The builder's 64-bit path (bucketed first sort, doubling rounds in chunks of whole groups, BWT and
    samples scattered from the ranks) forced on the same texts: the oracle's .bwt and .sa."""
    F = np.asarray(F, dtype=np.uint8)
    chunk = WIDE_CHUNK.get(name, 2 * len(F))
    st = galn_b200.index_text(F, str(tmp_path / "w"), sort_chunk=chunk)
    oracle.index_files(F, str(tmp_path / "o"))
    for ext in ("bwt", "sa"):
        assert _same(str(tmp_path / ("w." + ext)), str(tmp_path / ("o." + ext))), ext
    assert st["n"] == 2 * len(F)


def test_genome_shape_64bit_path_equals_32bit_path(tmp_path):
    """8 Mbp with repeat families, tandem repeats and N runs (16 M suffixes): the 64-bit path with a million
    suffixes per sort (many buckets, many chunks per round) writes the 32-bit path's files."""
    ref = synth.reference_genome(8_000_000, 31, n_contigs=5)
    fa = str(tmp_path / "ref.fa")
    synth.write_fasta(fa, ref)
    galn_b200.index_fasta(fa, str(tmp_path / "n"))
    F = oracle.forward_from_pac(str(tmp_path / "n.pac"))
    st = galn_b200.index_text(F, str(tmp_path / "w"), sort_chunk=1 << 20)
    for ext in ("bwt", "sa"):
        assert _same(str(tmp_path / ("w." + ext)), str(tmp_path / ("n." + ext))), ext
    assert st["rounds"] >= 2 and st["sorted_items"] > st["n"]


def test_genome_shape_against_fixture_builder(tmp_path):
    """8 Mbp with repeat families, tandem repeats and N runs: the fixture builder (prefix doubling on
    torch.sort, byte-identical to the reference builder on the golden genomes) gives the same five files."""
    ref = synth.reference_genome(8_000_000, 31, n_contigs=5)
    fa = str(tmp_path / "ref.fa")
    synth.write_fasta(fa, ref)
    index_build.build_index(fa, str(tmp_path / "fx"))
    st = galn_b200.index_fasta(fa, str(tmp_path / "gp"))
    for ext in EXTS:
        assert _same(str(tmp_path / ("gp." + ext)), str(tmp_path / ("fx." + ext))), ext
    assert st["rounds"] >= 2


def test_search_on_a_built_index(tmp_path):
    """The aDNA golden case searched on the index this builder wrote gives the reference's .sai bytes."""
    pre = str(tmp_path / "s")
    galn_b200.index_fasta(os.path.join(GOLDEN, "small", "ref.fa"), pre)
    meta = golden_cases()["adna"]
    p = case_paths("adna", meta)
    res = galn_b200.aln(galn_b200.Index(pre), meta["opts"], p["fq"])
    assert res.sai_bytes() == open(p["sai"], "rb").read()
