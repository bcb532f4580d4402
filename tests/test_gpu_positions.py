"""Genome positions of suffix-array rows on the GPU (samse's coordinate step: bwt_sa, bwa_sa2pos) against the
oracle, which is pinned to the suffix array itself (test_oracle.py): every row of the golden index, random
rows with random hit lengths, the rows of the reference's own .sai records, and a larger index with N runs."""
import os

import numpy as np
import pytest

import galn_b200
import oracle
from conftest import GOLDEN, case_paths, golden_cases
import fixture_index as index_build
from galn_b200 import build, synth

pytestmark = pytest.mark.gpu
PREFIX = os.path.join(GOLDEN, "small", "ref")


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()
    oracle.build()


@pytest.fixture(scope="module")
def small():
    ix = galn_b200.Index(PREFIX)
    ix.load_sa(PREFIX)
    o = oracle.Index(PREFIX + ".bwt")
    samples, intv = oracle.load_sa(PREFIX)
    return ix, o, samples, intv


def test_every_row(small):
    ix, o, samples, intv = small
    n_rows = int(o.L2[4]) + 1
    rows = np.arange(n_rows, dtype=np.uint64)
    np.testing.assert_array_equal(ix.bwt_sa(rows), oracle.bwt_sa(o, samples, intv, rows))


def test_random_rows_and_lengths(small):
    ix, o, samples, intv = small
    rng = np.random.default_rng(11)
    rows = rng.integers(0, int(o.L2[4]) + 1, 20000).astype(np.uint64)
    rl = rng.integers(1, 300, 20000).astype(np.int32)
    pos, strand = ix.sa2pos(rows, rl)
    opos, ostrand = oracle.sa2pos(o, samples, intv, rows, rl)
    np.testing.assert_array_equal(pos, opos)
    np.testing.assert_array_equal(strand, ostrand)


def test_rows_of_the_reference_sai(small):
    """Both ends of every hit interval of the reference's .sai for the aDNA case, with the hit's reference
    length (read length + deletions - insertions), as samse would ask."""
    ix, o, samples, intv = small
    meta = golden_cases()["adna"]
    p = case_paths("adna", meta)
    sai = oracle.read_sai(p["sai"])
    reads = galn_b200.read_fastq(p["fq"])
    lens = np.diff(reads.offset)
    recs = sai["records"]
    owner = np.repeat(np.arange(len(sai["n_aln"])), np.maximum(sai["n_aln"], 0))
    packed = recs["packed"].astype(np.uint64)
    n_ins = ((packed >> np.uint64(44)) & np.uint64(0x3ff)).astype(np.int32)
    n_del = ((packed >> np.uint64(54)) & np.uint64(0x3ff)).astype(np.int32)
    rl = (lens[owner] + n_del - n_ins).astype(np.int32)
    for col in ("k", "l"):
        rows = recs[col].astype(np.uint64)
        pos, strand = ix.sa2pos(rows, rl)
        opos, ostrand = oracle.sa2pos(o, samples, intv, rows, rl)
        np.testing.assert_array_equal(pos, opos)
        np.testing.assert_array_equal(strand, ostrand)


def test_larger_index_with_n_runs(tmp_path):
    ref = synth.reference_genome(2_000_000, 71)
    prefix = str(tmp_path / "g")
    index_build.build_from_reference(ref, prefix)
    ix = galn_b200.Index(prefix)
    ix.load_sa(prefix)
    o = oracle.Index(prefix + ".bwt")
    samples, intv = oracle.load_sa(prefix)
    rng = np.random.default_rng(12)
    rows = rng.integers(0, int(o.L2[4]) + 1, 30000).astype(np.uint64)
    rl = rng.integers(20, 200, 30000).astype(np.int32)
    pos, strand = ix.sa2pos(rows, rl)
    opos, ostrand = oracle.sa2pos(o, samples, intv, rows, rl)
    np.testing.assert_array_equal(pos, opos)
    np.testing.assert_array_equal(strand, ostrand)


def test_needs_samples_of_this_index(tmp_path):
    ix = galn_b200.Index(PREFIX)
    with pytest.raises(galn_b200.GalnError):
        ix.sa2pos(np.zeros(3, np.uint64), np.ones(3, np.int32))   # no .sa loaded
    with pytest.raises(galn_b200.GalnError):
        ix.load_sa(os.path.join(GOLDEN, "genome", "ref"))          # another index's samples
