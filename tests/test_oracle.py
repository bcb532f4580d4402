"""The oracle (oracle/galn_oracle.c, this project's CPU restatement of the search) against the golden
fixtures produced by the reference itself (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, case_paths, golden_cases
import fixture_index as index_build

CASES = golden_cases()


@pytest.fixture(scope="module", autouse=True)
def _built():
    oracle.build()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_sai(name, tmp_path):
    meta = CASES[name]
    p = case_paths(name, meta)
    ob = oracle.opt_bytes(oracle.parse_aln_args(meta["opts"]))
    expected = open(p["sai"], "rb").read()
    assert expected[4:68] == ob, "option block"
    reads = oracle.load_reads(p["fq"])
    idx = oracle.Index(p["prefix"] + ".bwt")
    res = oracle.aln(idx, ob, reads["query"], reads["off"], reads["len"], reads["batch"], 2)
    out = str(tmp_path / "o.sai")
    rc = res.write_sai(ob, out)
    assert rc == (4 if meta["rc"] == 4 else 0)
    assert open(out, "rb").read() == expected
    pr = np.load(p["per_read"])
    np.testing.assert_array_equal(res.n_aln, pr["n_aln"])
    np.testing.assert_array_equal(res.pops, pr["pops"])
    np.testing.assert_array_equal(res.trace, pr["trace"])
    np.testing.assert_array_equal(res.peak, pr["peak"])
    np.testing.assert_array_equal(reads["batch"], pr["batch"])
    np.testing.assert_array_equal(reads["len"], pr["len"])


def test_edge_reader_rules():
    meta = CASES["edge_default"]
    reads = oracle.load_reads(case_paths("edge_default", meta)["fq"])
    # the empty read is skipped and the malformed record dropped; the batch ends at the malformed record
    assert len(reads["len"]) == 55
    assert reads["batch"].max() == 1
    assert reads["len"].max() == 1000 and reads["len"].min() == 1


@pytest.mark.parametrize("refdir", ["small", "genome"])
def test_index_builder_matches_reference(refdir, tmp_path):
    src = os.path.join(os.path.dirname(__file__), "golden", refdir)
    prefix = str(tmp_path / "ix")
    index_build.build_index(os.path.join(src, "ref.fa"), prefix, "cpu")
    for ext in ("bwt", "sa", "pac", "ann", "amb"):
        assert open(prefix + "." + ext, "rb").read() == open(os.path.join(src, "ref." + ext), "rb").read(), ext


def test_cal_maxdiff_known_values():
    # bwa_cal_maxdiff(l, 0.02, fnr) for the read lengths and -n values of the workloads
    assert oracle.cal_maxdiff(100, 0.02, np.float32(0.04)) == 5
    assert oracle.cal_maxdiff(150, 0.02, np.float32(0.04)) == 6
    assert oracle.cal_maxdiff(50, 0.02, np.float32(0.01)) == 4
    assert oracle.cal_maxdiff(120, 0.02, np.float32(0.01)) == 7


_SA = {}


def _full_sa(prefix, tmp):
    """The suffix array of the index's text F.revcomp(F) (rows 0..n): F as the builder packs it (N bases
    replaced as bwa does), sorted by the fixture builder."""
    if prefix not in _SA:
        names, comments, seqs = index_build.read_fasta(prefix + ".fa")
        F = index_build.write_pac_ann_amb(str(tmp / "t"), names, comments, seqs)
        T = np.concatenate([F, (3 - F[::-1]).astype(np.uint8)])
        _SA[prefix] = index_build.suffix_array(T, "cpu")
    return _SA[prefix]


def test_oracle_bwt_sa_is_the_suffix_array(tmp_path):
    """The oracle's bwt_sa walk over the reference-built .bwt/.sa gives the suffix array itself at every row
    (row 0, the $ suffix, is bwa's -1)."""
    prefix = os.path.join(GOLDEN, "small", "ref")
    ix = oracle.Index(prefix + ".bwt")
    samples, intv = oracle.load_sa(prefix)
    sa = _full_sa(prefix, tmp_path)
    n = len(sa)
    got = oracle.bwt_sa(ix, samples, intv, range(n))
    assert got[0] == np.uint64(2**64 - 1)
    np.testing.assert_array_equal(got[1:], sa[1:].astype(np.uint64))


def test_oracle_sa2pos_rules(tmp_path):
    """bwa_sa2pos on top of bwt_sa: forward hits keep their coordinate (strand 1), reverse-half hits are
    mirrored to the first base (strand 0), hits across the forward/reverse boundary get -1."""
    prefix = os.path.join(GOLDEN, "small", "ref")
    ix = oracle.Index(prefix + ".bwt")
    samples, intv = oracle.load_sa(prefix)
    sa = _full_sa(prefix, tmp_path)
    l_pac = (len(sa) - 1) // 2
    rng = np.random.default_rng(3)
    rows = rng.integers(1, len(sa), 3000)
    rl = rng.integers(1, 200, 3000).astype(np.int32)
    pos, strand = oracle.sa2pos(ix, samples, intv, rows, rl)
    for k, r, p, st in zip(rows, rl, pos, strand):
        f = int(sa[k])
        if f < l_pac < f + r:
            assert p == np.uint64(2**64 - 1)
        elif f >= l_pac:
            g = 2 * l_pac - 1 - f
            assert st == 0 and int(p) == (0 if g + 1 < r else g - r + 1)
        else:
            assert st == 1 and int(p) == f
