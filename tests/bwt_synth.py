"""Test helper: a .bwt file in BWA's layout over random symbols, of any length (beyond 2^32 symbols too).

The symbols are not the BWT of any text; the file is only consistent in the way the occurrence layer reads
it: per 128 symbols four uint64 counts of each base before the block, then eight uint32 words of sixteen
2-bit symbols (first symbol in the top bits), the last block cut after the last symbol's word, then the four
totals; a 40-byte header of primary and L2[1..4] (= cumulative totals, L2[4] = the length). That is what the
occurrence layer (Occ of a row, the $ row `primary` skipped) needs, and what the tests of that layer across
the 2^32-symbol superblock boundary use.
"""
from __future__ import annotations

import numpy as np

M55 = np.uint32(0x55555555)


def _symbol_counts(words: np.ndarray) -> np.ndarray:
    """Per word, the number of symbols 0..3 among its 16 (shape (len, 4), uint8)."""
    lo = words & M55
    hi = (words >> np.uint32(1)) & M55
    c3 = np.bitwise_count(lo & hi)
    c1 = np.bitwise_count(lo & ~hi & M55)
    c2 = np.bitwise_count(~lo & hi & M55)
    out = np.empty((len(words), 4), np.uint8)
    out[:, 1], out[:, 2], out[:, 3] = c1, c2, c3
    out[:, 0] = 16 - c1 - c2 - c3
    return out


def _block_counts(words: np.ndarray, m: int) -> np.ndarray:
    """Symbols 0..3 in each run of 8 words (m runs; the words beyond 8 m, if any, form one more run)."""
    out = np.zeros((m + (len(words) > 8 * m), 4), np.int64)
    full = words[:8 * m].reshape(m, 8)
    lo = full & M55
    hi = (full >> np.uint32(1)) & M55
    out[:m, 3] = np.bitwise_count(lo & hi).sum(axis=1, dtype=np.int64)
    out[:m, 1] = np.bitwise_count(lo & ~hi).sum(axis=1, dtype=np.int64)
    out[:m, 2] = np.bitwise_count(~lo & hi & M55).sum(axis=1, dtype=np.int64)
    out[:m, 0] = 128 - out[:m, 1:].sum(axis=1)
    if len(words) > 8 * m:
        out[m] = _symbol_counts(words[8 * m:]).astype(np.int64).sum(axis=0)
    return out


def random_bwt(n: int, primary: int, seed: int, chunk_blocks: int = 1 << 21) -> np.ndarray:
    """The whole .bwt file (header and body) as uint32 words, for n pseudo-random symbols: a pool of
    chunk_blocks random 128-symbol blocks, laid down again and again, each time rotated by a random number
    of blocks (so the counts of a copy are the pool's, rotated, and a 2^32-symbol text takes seconds)."""
    assert 1 <= primary <= n
    rng = np.random.Generator(np.random.PCG64(seed))
    nw = (n + 15) // 16
    nb = (n + 127) // 128
    pb = min(chunk_blocks, nb)
    pool = rng.bit_generator.random_raw(4 * pb).view(np.uint32).reshape(pb, 8)
    pool_cnt = _block_counts(pool.reshape(-1), pb)
    # exclusive prefix of the pool's counts, doubled so that a rotation is one slice
    cum2 = np.zeros((2 * pb + 1, 4), np.int64)
    np.cumsum(np.concatenate([pool_cnt, pool_cnt]), axis=0, out=cum2[1:])
    out = np.empty(10 + 8 * (nb + 1) + nw, np.uint32)   # every word is written below
    body = out[10:]
    nfull_all = n // 128                                   # blocks of 128 symbols
    v32 = body[:16 * nfull_all].reshape(nfull_all, 16)
    v64 = body[:16 * nfull_all].view(np.uint64).reshape(nfull_all, 8)
    before = np.zeros(4, np.int64)
    tmp = np.empty((pb, 4), np.int64)     # one buffer for every copy's counts (fresh pages are slow)
    for b0 in range(0, nfull_all, pb):
        m = min(pb, nfull_all - b0)
        sh = int(rng.integers(0, pb))
        a = min(m, pb - sh)               # blocks taken from the pool before it wraps
        v32[b0:b0 + a, 8:] = pool[sh:sh + a]
        v32[b0 + a:b0 + m, 8:] = pool[:m - a]
        np.subtract(cum2[sh:sh + m], cum2[sh] - before, out=tmp[:m])
        v64[b0:b0 + m, :4] = tmp[:m].view(np.uint64)
        before = before + cum2[sh + m] - cum2[sh]
    if nfull_all < nb:                    # the last block, cut after its last word
        base = 16 * nfull_all
        rest = rng.bit_generator.random_raw(4).view(np.uint32)[:nw - 8 * nfull_all].copy()
        r = n % 16
        if r:
            rest[-1] &= np.uint32((0xffffffff << (32 - 2 * r)) & 0xffffffff)   # symbols past n are 0
        cnt = _symbol_counts(rest).astype(np.int64).sum(axis=0)
        if r:
            cnt[0] -= 16 - r                                                    # and not counted
        body[base:base + 8] = before.view(np.uint32)
        body[base + 8:base + 8 + len(rest)] = rest
        before = before + cnt
    body[-8:] = before.view(np.uint32)
    hdr = np.zeros(5, np.uint64)
    hdr[0] = primary
    hdr[1:] = np.cumsum(before)
    out[:10] = hdr.view(np.uint32)
    return out


def symbols(bwt_words: np.ndarray) -> np.ndarray:
    """The symbols of a random_bwt file (small sizes only): codes 0..3, length n."""
    hdr = bwt_words[:10].view(np.uint64)
    n = int(hdr[4])
    body = bwt_words[10:]
    nb = (n + 127) // 128
    out = np.empty(nb * 128, np.uint8)
    for b in range(nb):
        ws = body[16 * b + 8:16 * b + 16]
        for j, w in enumerate(ws):
            if 128 * b + 16 * j >= n:
                break
            for t in range(16):
                out[128 * b + 16 * j + t] = (int(w) >> (30 - 2 * t)) & 3
    return out[:n]


def occ_brute(sym: np.ndarray, primary: int, rows) -> np.ndarray:
    """Occ of the four bases at each row, counted from the symbols ($ row skipped; ~0 = row -1)."""
    cum = np.zeros((len(sym) + 1, 4), np.uint64)
    for c in range(4):
        cum[1:, c] = np.cumsum(sym == c)
    out = np.zeros((len(rows), 4), np.uint64)
    for i, k in enumerate(rows):
        k = int(k)
        if k == (1 << 64) - 1:
            continue
        p = k - (k >= primary)
        out[i] = cum[p + 1]
    return out
