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


def test_heavy_request_held_back_by_stack_memory(ix):
    """Admission by stack memory: with a budget that holds a large light request and a small one, a request
    whose options need a much deeper stack (-m 50,000,000) is held back while light requests submitted after
    it are admitted; every result still equals the request searched alone."""
    plain = galn_b200.read_fastq(case_paths("plain", CASES["plain"])["fq"])
    adna = galn_b200.read_fastq(case_paths("adna", CASES["adna"])["fq"])
    seqs = [bytes(plain.seq[plain.offset[i]:plain.offset[i + 1]]) for i in range(len(plain))]
    big = galn_b200.Reads.from_strings(seqs * 40)                      # 80,000 reads, default options
    small = galn_b200.Reads(plain.seq, plain.offset)
    heavy_opts = list(CASES["adna"]["opts"]) + ["-m", "50000000"]
    heavy = galn_b200.Reads(adna.seq, adna.offset)
    reqs = [("L1", [], big), ("H", heavy_opts, heavy), ("L2", [], small), ("L3", [], small)]
    alone = {name: galn_b200.aln(ix, opts, reads).sai_bytes() for name, opts, reads in reqs}
    probe = galn_b200.Server(ix)
    need = {name: probe.stack_need(opts, reads) for name, opts, reads in reqs}
    probe.close()
    assert need["H"] > need["L2"] + (1 << 20)
    budget = need["L1"] + need["L2"] + (1 << 20)
    srv = galn_b200.Server(ix, stack_bytes=budget)
    try:
        ids = {name: srv.submit(opts, reads) for name, opts, reads in reqs}
        got = {name: srv.wait(rid).sai_bytes() for name, rid in ids.items()}
        order = srv.admissions()
        mem = srv.memory()
    finally:
        srv.close()
    for name in alone:
        assert got[name] == alone[name], name
    assert mem["budget"] == budget and mem["peak"] <= budget
    assert mem["held_back"] >= 1
    assert order.index(ids["H"]) > order.index(ids["L2"]), "the heavy request was not held back"
