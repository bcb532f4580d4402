"""The occurrence layer and the search on an index of more than 2^32 symbols (the genome-scale text length,
6.2 x 10^9 symbols for 3.1 Gbp, crosses it): counts are kept relative to 2^32-symbol superblocks (occ64) and
2^25-block superblocks (occ80), so rows on both sides of each boundary are checked against the oracle's
count over the .bwt file, and searches whose intervals lie above 2^32 give the oracle's results. The index
is 1.5 x 2^32 + 77 pseudo-random symbols in BWA's .bwt layout (about 3.2 GB; tests/bwt_synth.py), the $ row
above 2^32 too."""
import numpy as np
import pytest

import bwt_synth
import galn_b200
import oracle
from galn_b200 import build

pytestmark = pytest.mark.gpu
N = (3 << 31) + 77
PRIMARY = 4_500_000_123
OCC80_SUPER = 80 << 25          # symbols per occ80 superblock
COMP = np.array([3, 2, 1, 0], np.uint8)


@pytest.fixture(scope="module")
def big():
    build.build()
    oracle.build()
    words = bwt_synth.random_bwt(N, PRIMARY, seed=5)   # the .bwt file's image, shared by both sides
    ox = oracle.Index(file_words=words)
    ix = galn_b200.Index(bwt_bytes=words)
    yield ix, ox, words
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
    ix, ox, _ = big
    assert ix.info()["seq_len"] == N
    rows = _rows()
    np.testing.assert_array_equal(ix.occ(rows, layout), ox.occ4(rows))


def _walk_reads(words, ox, n, length, seed):
    """Reads that occur in the index: from random rows, `length` steps of the inverse suffix-array walk
    (row r holds symbol c = BWT[r]; the previous row is C[c] + Occ(c, r)) spell a substring of the text the
    BWT encodes; the read is its reverse complement, which aln searches backwards as that substring."""
    rng = np.random.default_rng(seed)
    L2 = words[:10].view(np.uint64)
    C = np.array([0, L2[1], L2[2], L2[3]], np.uint64)
    body = words[10:]
    rows = rng.integers(0, N + 1, size=4 * n, dtype=np.uint64)
    rows = rows[rows != PRIMARY][:n]
    sym = np.zeros((n, length), np.uint8)
    ok = np.ones(n, bool)
    for t in range(length):
        ok &= rows != PRIMARY
        r = np.where(rows == PRIMARY, 0, rows)
        p = r - (r > PRIMARY)
        w = body[(p >> 7) * 16 + 8 + ((p & 127) >> 4)]
        c = ((w >> (30 - 2 * (p & 15)).astype(np.uint32)) & 3).astype(np.uint8)
        sym[:, length - 1 - t] = c             # the text runs ... c_t ... c_1, the suffix of row r after it
        occ = ox.occ4(r)
        rows = C[c] + occ[np.arange(n), c]
    sub = sym[ok]
    reads = COMP[sub[:, ::-1]]                 # reverse complement of the substring
    return np.frombuffer(b"ACGT", np.uint8)[reads.reshape(-1)].copy(), len(sub)


@pytest.mark.parametrize("layout", [64, 80])
def test_search_above_2_32(big, layout):
    """Reads spelled by the index itself and random reads, 40 bp with -n 4 -l 1024 (the symbols are not a
    text closed under reverse complement, so the width bound of longer reads would prune every search):
    per read n_aln, pops, trace and records equal the oracle's, and hits lie on both sides of 2^32."""
    ix, ox, words = big
    L = 40
    opts = ["-n", "4", "-l", "1024"]
    seq_hit, n_hit = _walk_reads(words, ox, 1500, L, 13)
    rng = np.random.default_rng(11)
    seq_rand = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, size=500 * L)].copy()
    seq = np.concatenate([seq_hit, seq_rand])
    n = n_hit + 500
    off = np.arange(n + 1, dtype=np.int64) * L
    reads = galn_b200.Reads(seq, off)
    ix.set_occ_layout(layout)
    res = galn_b200.aln(ix, opts, reads, galn_b200.GALN_ENGINE_PERSISTENT)
    ix.set_occ_layout(64)
    query = oracle.encode_queries(seq, off)
    o = oracle.aln(ox, oracle.opt_bytes(oracle.parse_aln_args(opts)), query, off, np.full(n, L, np.int32),
                   oracle.batches_for(n))
    np.testing.assert_array_equal(res.n_aln, o.n_aln)
    np.testing.assert_array_equal(res.pops, o.pops)
    np.testing.assert_array_equal(res.trace, o.trace)
    np.testing.assert_array_equal(res.records, o.records)
    assert (res.n_aln[:n_hit] > 0).mean() > 0.9
    k = res.records["k"]
    assert (k >= (1 << 32)).any() and (k < (1 << 32)).any()
