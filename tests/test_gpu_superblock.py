"""The occurrence layer and the search on an index of more than 2^32 symbols (the genome-scale text length,
6.2 x 10^9 symbols for 3.1 Gbp, crosses it): counts are kept relative to 2^32-symbol superblocks (occ64) and
2^25-block superblocks (occ80), so rows on both sides of each boundary are checked against the oracle's
count over the .bwt file, and a search whose intervals live above 2^32 gives the oracle's results. The
index is 2^32 + 2^22 + 77 random symbols in BWA's .bwt layout (about 2.15 GB; tests/bwt_synth.py)."""
import os

import numpy as np
import pytest

import bwt_synth
import galn_b200
import oracle
from galn_b200 import build

pytestmark = pytest.mark.gpu
N = (1 << 32) + (1 << 22) + 77
PRIMARY = 3_000_000_123
OCC80_SUPER = 80 << 25          # symbols per occ80 superblock


@pytest.fixture(scope="module")
def big():
    build.build()
    oracle.build()
    words = bwt_synth.random_bwt(N, PRIMARY, seed=5)   # the .bwt file's image, shared by both sides
    ox = oracle.Index(file_words=words)
    ix = galn_b200.Index(bwt_bytes=words)
    yield ix, ox
    ix.close()


def _rows():
    """Rows whose $-free positions sit at every superblock boundary and block edge near it, the $ row, the
    ends, and random rows."""
    pos = []
    for b in (1 << 32, OCC80_SUPER, 2 * OCC80_SUPER, PRIMARY):
        pos += list(range(b - 200, b + 200))
    pos += list(range(0, 300)) + list(range(N - 300, N))
    pos = np.array(sorted(set(p for p in pos if 0 <= p < N)), np.uint64)
    rows = pos + (pos >= PRIMARY).astype(np.uint64)
    rng = np.random.default_rng(9)
    extra = np.array([PRIMARY, N, (1 << 64) - 1], np.uint64)
    return np.concatenate([rows, extra, rng.integers(0, N + 1, size=50_000, dtype=np.uint64)])


@pytest.mark.parametrize("layout", [64, 80])
def test_occ_across_superblocks(big, layout):
    ix, ox = big
    assert ix.info()["seq_len"] == N
    rows = _rows()
    np.testing.assert_array_equal(ix.occ(rows, layout), ox.occ4(rows))


@pytest.mark.parametrize("layout", [64, 80])
def test_search_above_2_32(big, layout):
    """Random 100 bp reads searched with default options: per read n_aln, pops and trace equal the
    oracle's, and some records' intervals lie above 2^32."""
    ix, ox = big
    rng = np.random.default_rng(11)
    n, L = 2000, 100
    codes = rng.integers(0, 4, size=n * L, dtype=np.uint8)
    seq = np.frombuffer(b"ACGT", np.uint8)[codes]
    off = np.arange(n + 1, dtype=np.int64) * L
    reads = galn_b200.Reads(seq.copy(), off)
    ix.set_occ_layout(layout)
    res = galn_b200.aln(ix, [], reads, galn_b200.GALN_ENGINE_PERSISTENT)
    ix.set_occ_layout(64)
    query = oracle.encode_queries(seq, off)
    o = oracle.aln(ox, oracle.opt_bytes(oracle.parse_aln_args([])), query, off, np.full(n, L, np.int32),
                   oracle.batches_for(n))
    np.testing.assert_array_equal(res.n_aln, o.n_aln)
    np.testing.assert_array_equal(res.pops, o.pops)
    np.testing.assert_array_equal(res.trace, o.trace)
    assert (res.records["k"] >= (1 << 32)).any()
