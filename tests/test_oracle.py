"""The oracle (oracle/galn_oracle.c, this project's CPU restatement of the search) against the golden
fixtures produced by the reference itself (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import oracle
from conftest import case_paths, golden_cases
from galn_b200 import index_build

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
