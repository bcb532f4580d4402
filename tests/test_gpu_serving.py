"""The serving loop (continuous batching): requests with their own options and batch boundaries share
steps on the device, and every request's .sai, pop counts and trace hashes are the same alone, mixed with
others, split over many steps, and submitted from several host threads; they equal the reference's golden
files where those exist."""
import os
import threading

import numpy as np
import pytest

import galn_b200
from conftest import GOLDEN, case_paths, golden_cases

pytestmark = pytest.mark.gpu
CASES = golden_cases()
SMALL = [n for n, m in CASES.items() if m["ref"] == "small"]


@pytest.fixture(scope="module")
def ix():
    return galn_b200.Index(os.path.join(GOLDEN, "small", "ref"))


def _requests():
    out = []
    for name in sorted(SMALL):
        meta = CASES[name]
        out.append((name, meta["opts"], galn_b200.read_fastq(case_paths(name, meta)["fq"])))
    return out


@pytest.mark.parametrize("step,fill", [(1024, 0), (4096, 0), (1 << 18, 0), (4096, 4096), (1 << 18, 1 << 18)])
def test_mixed_requests_equal_alone_and_golden(ix, step, fill):
    reqs = _requests()
    alone = {name: galn_b200.aln(ix, opts, reads) for name, opts, reads in reqs}
    srv = galn_b200.Server(ix, step_reads=step, max_active=64, fill_reads=fill)
    try:
        ids = [(name, srv.submit(opts, reads)) for name, opts, reads in reqs]
        ids += [(name + "#2", srv.submit(opts, reads)) for name, opts, reads in reqs]   # every request twice
        got = {name: srv.wait(rid) for name, rid in ids}
        st = srv.stats()
    finally:
        srv.close()
    assert st["requests"] == len(ids) and st["steps"] >= 1
    for name, opts, reads in reqs:
        for key in (name, name + "#2"):
            r = got[key]
            assert r.sai_bytes() == alone[name].sai_bytes(), key
            np.testing.assert_array_equal(r.pops, alone[name].pops)
            np.testing.assert_array_equal(r.trace, alone[name].trace)
            assert r.sai_bytes() == open(case_paths(name, CASES[name])["sai"], "rb").read(), key


def test_submit_from_many_threads(ix):
    reqs = _requests()
    alone = {name: galn_b200.aln(ix, opts, reads).sai_bytes() for name, opts, reads in reqs}
    srv = galn_b200.Server(ix, step_reads=2048)
    results, errors = {}, []

    def client(k):
        try:
            for name, opts, reads in reqs[k::3]:
                rid = srv.submit(opts, reads)
                results[(k, name)] = srv.wait(rid).sai_bytes()
        except Exception as e:   # noqa: BLE001
            errors.append(e)

    th = [threading.Thread(target=client, args=(k,)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    srv.close()
    assert not errors
    for (k, name), b in results.items():
        assert b == alone[name]


def test_empty_request(ix):
    srv = galn_b200.Server(ix)
    rid = srv.submit([], galn_b200.Reads.from_strings([]))
    assert len(srv.wait(rid)) == 0
    srv.close()
