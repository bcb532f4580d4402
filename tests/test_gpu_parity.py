"""The CUDA path against the reference: byte-identical .sai, and per read the same n_aln, pop count and
trace hash as the reference's search (golden fixtures), for both engines and when reads migrate between
tiers; larger synthetic cases against the oracle."""
import os

import numpy as np
import pytest

import galn_b200
import oracle
from conftest import GOLDEN, case_paths, golden_cases
import fixture_index as index_build
from galn_b200 import build, synth

pytestmark = pytest.mark.gpu
CASES = golden_cases()
ENGINES = [galn_b200.GALN_ENGINE_PLAIN, galn_b200.GALN_ENGINE_PERSISTENT]


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()
    oracle.build()


_ix_cache = {}


def index_for(refdir):
    if refdir not in _ix_cache:
        _ix_cache[refdir] = galn_b200.Index(os.path.join(GOLDEN, refdir, "ref"))
    return _ix_cache[refdir]


@pytest.mark.parametrize("occ", [64, 80])
@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_case(name, engine, occ):
    meta = CASES[name]
    p = case_paths(name, meta)
    ix = index_for(meta["ref"])
    ix.set_occ_layout(occ)
    res = galn_b200.aln(ix, meta["opts"], p["fq"], engine)
    ix.set_occ_layout(64)
    expected = open(p["sai"], "rb").read()
    assert res.sai_bytes() == expected
    pr = np.load(p["per_read"])
    np.testing.assert_array_equal(res.n_aln, pr["n_aln"])
    np.testing.assert_array_equal(res.pops, pr["pops"])
    np.testing.assert_array_equal(res.trace, pr["trace"])


@pytest.mark.parametrize("occ", [64, 80])
@pytest.mark.parametrize("trace", [True, False])
@pytest.mark.parametrize("warp", [(True, 8192), (True, 32), (False, 32)])
@pytest.mark.parametrize("caps", [(16, 1, 64, 16, 1), (64, 2, 256, 128, 2), (300, 4, 128, 1000, 3)])
def test_tier_migration_gives_same_bytes(caps, warp, trace, occ):
    """Tiny first- and second-tier capacities push many reads through every tier (the warp tier with a
    normal and a tiny arena, or without it), in both occurrence layouts; the bytes and traces stay the
    reference's and the per-read block fetches are the oracle's count for the layout."""
    ix = galn_b200.Index(os.path.join(GOLDEN, "small", "ref"))
    t0_cap, t0_aln, block, t1_cap, t1_aln = caps
    ix.set_tuning(t0_cap, t0_aln, block, t1_cap, t1_aln, keep_stats=True)
    ix.set_warp_tier(*warp)
    ix.set_trace(trace)
    ix.set_occ_layout(occ)
    for name in ("adna", "divergent", "edge_nonstop", "tiny_queue"):
        meta = CASES[name]
        p = case_paths(name, meta)
        rd = oracle.load_reads(p["fq"])
        o = oracle.aln(oracle.Index(os.path.join(GOLDEN, meta["ref"], "ref.bwt")),
                       oracle.opt_bytes(oracle.parse_aln_args(meta["opts"])), rd["query"], rd["off"], rd["len"],
                       rd["batch"], 4)
        for engine in ENGINES:
            res = galn_b200.aln(ix, meta["opts"], p["fq"], engine)
            assert res.sai_bytes() == open(p["sai"], "rb").read(), (name, engine)
            pr = np.load(p["per_read"])
            if trace:
                np.testing.assert_array_equal(res.trace, pr["trace"])
            np.testing.assert_array_equal(res.pops, pr["pops"])
            prof = ix.last_profile(len(res))
            np.testing.assert_array_equal(prof["fetch"].astype(np.uint64), o.fetch64 if occ == 64 else o.fetch80)
        st = ix.last_stats()
        assert st["tiers"] >= 2 or name in ("edge_nonstop", "tiny_queue")


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("trace", [True, False])
def test_fused_and_two_launch_forms_give_same_bytes(fused, trace):
    """The persistent engine with the first and warp tiers as one launch (heavy reads handed over through a
    device queue while light ones run) and as two launches: the reference's bytes and the same pops, with a
    tiny first tier so that most reads cross over."""
    ix = galn_b200.Index(os.path.join(GOLDEN, "small", "ref"))
    ix.set_fused(fused)
    ix.set_trace(trace)
    for cap in (16, 256):
        ix.set_tuning(cap, 2, 128, 65536, 1024)
        for name in ("adna", "divergent", "edge_nonstop", "edge_loggap", "plain", "tiny_queue"):
            meta = CASES[name]
            p = case_paths(name, meta)
            res = galn_b200.aln(ix, meta["opts"], p["fq"], galn_b200.GALN_ENGINE_PERSISTENT)
            assert res.sai_bytes() == open(p["sai"], "rb").read(), (name, cap)
            pr = np.load(p["per_read"])
            np.testing.assert_array_equal(res.pops, pr["pops"])
            if trace:
                np.testing.assert_array_equal(res.trace, pr["trace"])
            assert ix.last_profile()["fused"] == fused


@pytest.mark.parametrize("order", [0, 1])
def test_warp_order_keeps_bytes(order):
    """The order in which heavy reads reach the warp tier (by max_diff and length, or by the first tier's
    pops at overflow) changes nothing in the results."""
    ix = galn_b200.Index(os.path.join(GOLDEN, "small", "ref"))
    ix.set_fused(False)
    ix.set_warp_order(order)
    ix.set_tuning(16, 2, 128, 65536, 1024)
    for name in ("adna", "divergent", "edge_nonstop"):
        meta = CASES[name]
        p = case_paths(name, meta)
        res = galn_b200.aln(ix, meta["opts"], p["fq"], galn_b200.GALN_ENGINE_PERSISTENT)
        assert res.sai_bytes() == open(p["sai"], "rb").read(), name
        np.testing.assert_array_equal(res.trace, np.load(p["per_read"])["trace"])


@pytest.mark.parametrize("wait_ns", [0, 20_000])
def test_warp_wait_running_out_gives_same_bytes(wait_ns):
    """The big-arena warps' bounded wait for queued reads, made to run out: at 0 every wait gives up at
    once and the host searches every queued read again in a second launch; at 20 us some waits run out and
    the reads left in the queue go to the second launch. Bytes, pops and traces stay the reference's."""
    ix = galn_b200.Index(os.path.join(GOLDEN, "small", "ref"))
    ix.set_tuning(16, 1, 64, 16, 1)
    ix.set_warp_tier(True, 32)          # a tiny arena: heavy reads outgrow it and are queued
    ix.set_warp_wait(wait_ns)
    queued, gave_up = 0, 0
    for name in ("adna", "divergent", "edge_nonstop", "tiny_queue"):
        meta = CASES[name]
        p = case_paths(name, meta)
        res = galn_b200.aln(ix, meta["opts"], p["fq"], galn_b200.GALN_ENGINE_PERSISTENT)
        assert res.sai_bytes() == open(p["sai"], "rb").read(), name
        pr = np.load(p["per_read"])
        np.testing.assert_array_equal(res.pops, pr["pops"])
        np.testing.assert_array_equal(res.trace, pr["trace"])
        q = ix.last_warp_queue()
        queued += q["queued"]
        gave_up += int(q["gave_up"])
    assert queued > 0, "no read was queued for a big-arena warp"
    if wait_ns == 0:
        assert gave_up > 0, "no wait ran out"


@pytest.mark.parametrize("occ", [64, 80])
def test_fetch_counts_match_oracle(occ):
    """The per-read count of 32-byte index blocks the kernels read is the oracle's algorithmic count, for
    the layout in use."""
    ix = galn_b200.Index(os.path.join(GOLDEN, "small", "ref"))
    ix.set_tuning(keep_stats=True)
    ix.set_occ_layout(occ)
    for name in ("plain", "adna", "edge_seed"):
        meta = CASES[name]
        p = case_paths(name, meta)
        res = galn_b200.aln(ix, meta["opts"], p["fq"])
        prof = ix.last_profile(len(res))
        rd = oracle.load_reads(p["fq"])
        o = oracle.aln(oracle.Index(meta and os.path.join(GOLDEN, meta["ref"], "ref.bwt")),
                       oracle.opt_bytes(oracle.parse_aln_args(meta["opts"])), rd["query"], rd["off"], rd["len"],
                       rd["batch"], 4)
        np.testing.assert_array_equal(prof["fetch"].astype(np.uint64), o.fetch64 if occ == 64 else o.fetch80)


def test_index_from_memory():
    data = open(os.path.join(GOLDEN, "small", "ref.bwt"), "rb").read()
    ix = galn_b200.Index(bwt_bytes=data)
    meta = CASES["plain"]
    p = case_paths("plain", meta)
    res = galn_b200.aln(ix, meta["opts"], p["fq"])
    assert res.sai_bytes() == open(p["sai"], "rb").read()


def _compare_with_oracle(prefix, reads, opts, engines=ENGINES, trace=True, layouts=(64,)):
    ix = galn_b200.Index(prefix)
    ix.set_trace(trace)
    q = oracle.encode_queries(reads.seq, reads.offset)
    batch = reads.batch if reads.batch is not None else oracle.batches_for(len(reads))
    o = oracle.aln(oracle.Index(prefix + ".bwt"), oracle.opt_bytes(oracle.parse_aln_args(opts)), q, reads.offset,
                   np.diff(reads.offset).astype(np.int32), batch, 0)
    for occ in layouts:
        ix.set_occ_layout(occ)
        for engine in engines:
            res = galn_b200.aln(ix, opts, reads, engine)
            np.testing.assert_array_equal(res.n_aln, o.n_aln)
            np.testing.assert_array_equal(res.pops, o.pops)
            if trace:
                np.testing.assert_array_equal(res.trace, o.trace)
            np.testing.assert_array_equal(res.rec_offset, o.rec_off)
            assert res.records.tobytes() == o.records.tobytes()


@pytest.fixture(scope="module")
def adna_index(tmp_path_factory):
    d = tmp_path_factory.mktemp("adna")
    ref = synth.reference_adna(2_000_000, 21)
    index_build.build_from_reference(ref, str(d / "ref"))
    return ref, str(d / "ref")


@pytest.mark.parametrize("trace", [True, False])
@pytest.mark.parametrize("workload,n,seed", [("adna", 40_000, 31), ("divergent", 300, 32), ("plain", 20_000, 33)])
def test_synthetic_against_oracle(adna_index, workload, n, seed, trace):
    ref, prefix = adna_index
    if workload == "adna":
        r = synth.simulate_reads(ref, n, seed, synth.adna_lengths, sub_rate=0.005, random_frac=0.03, deaminate=0.3)
        opts = synth.ADNA_OPTS
    elif workload == "divergent":
        r = synth.simulate_reads(ref, n, seed, 100, sub_rate=0.04, indel_rate=0.005)
        opts = synth.DIVERGENT_OPTS
    else:
        r = synth.simulate_reads(ref, n, seed, 100, sub_rate=0.01, indel_rate=0.001, random_frac=0.02)
        opts = []
    reads = galn_b200.Reads(r.ascii(), r.off)
    _compare_with_oracle(prefix, reads, opts, trace=trace, layouts=(64, 80) if not trace else (64,))


def test_batch_boundary_mixed_lengths(adna_index):
    """0x40000 short reads then longer ones: the first bwa batch gets a smaller max_diff and a clamped
    max_gapo (-n 0.01 -o 3), the second batch its own options."""
    ref, prefix = adna_index
    a = synth.simulate_reads(ref, 0x40000, 41, 16, sub_rate=0.01, random_frac=0.02)
    b = synth.simulate_reads(ref, 3000, 42, lambda rng, m: rng.integers(30, 150, size=m), sub_rate=0.01,
                             random_frac=0.02)
    seq = np.concatenate([a.ascii(), b.ascii()])
    off = np.concatenate([a.off[:-1], b.off + a.off[-1]])
    reads = galn_b200.Reads(seq, off)
    _compare_with_oracle(prefix, reads, ["-n", "0.01", "-o", "3"], [galn_b200.GALN_ENGINE_PERSISTENT])


def test_genome_with_ambiguous_bases(tmp_path):
    ref = synth.reference_genome(3_000_000, 51)
    prefix = str(tmp_path / "g")
    index_build.build_from_reference(ref, prefix)
    r = synth.simulate_reads(ref, 8000, 52, 150, sub_rate=lambda x: 0.001 + 0.014 * x, indel_rate=0.0005)
    _compare_with_oracle(prefix, galn_b200.Reads(r.ascii(), r.off), [], layouts=(64, 80))


def test_empty_and_single_read():
    ix = index_for("small")
    res = galn_b200.aln(ix, [], galn_b200.Reads.from_strings([]))
    assert len(res) == 0
    res = galn_b200.aln(ix, [], galn_b200.Reads.from_strings(["ACGTTGCA"]))
    assert len(res) == 1


def test_autotune_and_graph_keep_bytes():
    """The autotuner's choice and the CUDA-graph launch of the first tier change speed only."""
    ix = galn_b200.Index(os.path.join(GOLDEN, "small", "ref"))
    meta = CASES["adna"]
    p = case_paths("adna", meta)
    reads = galn_b200.read_fastq(p["fq"])
    tune = ix.autotune(meta["opts"], reads)
    assert tune["t0_cap"] in (256, 512, 1024, 2048, 4096) and tune["block"] in (128, 256)
    assert tune["occ"] in (64, 80)
    for _ in range(2):   # the second run updates the instantiated graph
        res = galn_b200.aln(ix, meta["opts"], reads)
        assert res.sai_bytes() == open(p["sai"], "rb").read()
        assert ix.last_stats()["graph_launches"] >= 1
