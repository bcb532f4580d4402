"""BWA-format index files for a FASTA reference: <prefix>.pac/.ann/.amb/.bwt/.sa, in Python on torch.

The library's own builder is `galn index` (galn_index_build_fasta: the suffix sort in CUDA kernels); this
module is a second, independent implementation that the tests compare it with. The files follow `bwa
index` 0.7.19 byte for byte (the BWT of a text is unique, so any correct suffix sort gives the same .bwt):

  * text T = F . revcomp(F), F the forward 2-bit sequence; an ambiguous base becomes lrand48() & 3 from
    a generator seeded with srand48(11), drawn in sequence order; runs of the same ambiguous character
    are the .amb holes (the rule of bwa's bntseq.c add1/bns_fasta2bntseq);
  * .pac = F packed 4 bases per byte, most significant pair first, then a 0 byte if l_pac % 4 == 0, then
    a byte holding l_pac % 4;
  * .bwt = primary, L2[1..4] (uint64 each), then per 128 symbols 4 x uint64 occurrence counts before
    the block and 8 x uint32 words of 2-bit symbols (most significant pair first), then 4 x uint64
    totals; the $ row `primary` is left out of the symbols;
  * .sa = primary, L2[1..4], 32, n, then SA[32], SA[64], ... over the n+1 rows (row 0 is $).

The suffix array is built by prefix doubling on top of torch.sort, on the GPU when one is present and
on the host otherwise. The first round sorts 21-symbol prefixes packed 3 bits per symbol; each later
round sorts (rank[i], rank[i+h]) pairs and doubles h until all ranks are distinct.
"""
from __future__ import annotations

import os

import numpy as np

NT4 = np.full(256, 4, dtype=np.uint8)
for _i, _c in enumerate(b"ACGT"):
    NT4[_c] = _i
    NT4[_c + 32] = _i

_LCG_A = 0x5DEECE66D
_LCG_C = 0xB
_M48 = (1 << 48) - 1


class Lrand48:
    """POSIX lrand48: x <- (0x5DEECE66D x + 11) mod 2^48, returns x >> 17; srand48(s) sets x = s<<16 | 0x330E."""

    def __init__(self, seed: int):
        self.x = ((seed & 0xFFFFFFFF) << 16) | 0x330E

    def draws(self, n: int) -> np.ndarray:
        """The next n values of lrand48() & 3."""
        out = np.empty(n, dtype=np.uint8)
        x = self.x
        for i in range(n):
            x = (_LCG_A * x + _LCG_C) & _M48
            out[i] = (x >> 17) & 3
        self.x = x
        return out


def read_fasta(path: str):
    """(names, comments, raw sequence bytes) of each record; header = name up to the first white space,
    the rest of the line (after that one character) is the comment."""
    import gzip
    opener = gzip.open if path.endswith(".gz") else open
    with opener(path, "rb") as f:
        data = f.read()
    names, comments, seqs = [], [], []
    for rec in data.split(b"\n>"):
        if not rec:
            continue
        if rec.startswith(b">"):
            rec = rec[1:]
        nl = rec.find(b"\n")
        head, body = (rec, b"") if nl < 0 else (rec[:nl], rec[nl + 1:])
        head = head.rstrip(b"\r")
        parts = head.split(None, 1)
        names.append(parts[0].decode() if parts else "")
        comments.append(parts[1].decode() if len(parts) > 1 else "")
        seqs.append(body.replace(b"\n", b"").replace(b"\r", b""))
    return names, comments, seqs


def write_pac_ann_amb(prefix: str, names, comments, seqs) -> np.ndarray:
    """Writes .pac/.ann/.amb; returns the forward sequence as codes 0..3 (ambiguous bases replaced)."""
    rng = Lrand48(11)
    fwd = []
    holes = []           # (offset, len, char)
    n_ambs = []
    offset = 0
    for s in seqs:
        raw = np.frombuffer(s, dtype=np.uint8)
        codes = NT4[raw].copy()
        amb = np.nonzero(codes >= 4)[0]
        cnt = 0
        if len(amb):
            codes[amb] = rng.draws(len(amb))
            # a hole continues while the same ambiguous character repeats at consecutive positions
            prev_same = np.zeros(len(amb), dtype=bool)
            prev_same[1:] = (amb[1:] == amb[:-1] + 1) & (raw[amb[1:]] == raw[amb[:-1]])
            if amb[0] > 0 and raw[amb[0] - 1] == raw[amb[0]]:
                prev_same[0] = True   # cannot happen: the previous base is not ambiguous
            starts = np.nonzero(~prev_same)[0]
            ends = np.append(starts[1:], len(amb))
            for a, b in zip(starts, ends):
                holes.append((offset + int(amb[a]), int(b - a), chr(raw[amb[a]])))
            cnt = len(starts)
        n_ambs.append(cnt)
        fwd.append(codes)
        offset += len(s)
    F = np.concatenate(fwd) if fwd else np.zeros(0, np.uint8)
    l_pac = len(F)
    pad = (-l_pac) % 4
    Fp = np.concatenate([F, np.zeros(pad, np.uint8)]).reshape(-1, 4)
    pac = (Fp[:, 0] << 6 | Fp[:, 1] << 4 | Fp[:, 2] << 2 | Fp[:, 3]).astype(np.uint8)
    tail = (b"\x00" if l_pac % 4 == 0 else b"") + bytes([l_pac % 4])
    with open(prefix + ".pac", "wb") as f:
        f.write(pac.tobytes() + tail)
    with open(prefix + ".ann", "w") as f:
        f.write(f"{l_pac} {len(seqs)} 11\n")
        off = 0
        for name, com, s, na in zip(names, comments, seqs, n_ambs):
            f.write(f"0 {name} {com if com else '(null)'}\n")
            f.write(f"{off} {len(s)} {na}\n")
            off += len(s)
    with open(prefix + ".amb", "w") as f:
        f.write(f"{l_pac} {len(seqs)} {len(holes)}\n")
        for o, ln, ch in holes:
            f.write(f"{o} {ln} {ch}\n")
    return F


def suffix_array(T: np.ndarray, device: str | None = None) -> np.ndarray:
    """SA of T$ over its n+1 rows (row 0 is the $ suffix, position n), as int64."""
    import torch
    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    n = len(T)
    N = n + 1
    K = 21
    codes = torch.zeros(N + K, dtype=torch.int64, device=device)
    codes[:n] = torch.from_numpy(T.astype(np.int64)).to(device) + 1
    key = torch.zeros(N, dtype=torch.int64, device=device)
    for t in range(K):
        key = (key << 3) | codes[t:t + N]
    del codes
    h = K
    idx = torch.arange(N, dtype=torch.int64, device=device)
    while True:
        vals, order = torch.sort(key)
        new_group = torch.ones(N, dtype=torch.bool, device=device)
        new_group[1:] = vals[1:] != vals[:-1]
        start = torch.where(new_group, idx, torch.zeros_like(idx))
        start = torch.cummax(start, dim=0).values
        rank = torch.empty(N, dtype=torch.int64, device=device)
        rank[order] = start
        n_groups = int(new_group.sum())
        del vals, new_group, start
        if n_groups == N:
            return order.cpu().numpy()
        del order
        nxt = torch.zeros(N, dtype=torch.int64, device=device)
        if h < N:
            nxt[:N - h] = rank[h:] + 1
        key = rank * (N + 1) + nxt
        del rank, nxt
        h *= 2


def pack_bwt(L: np.ndarray):
    """bwa's .bwt body for the n symbols L (0..3, $ removed): (uint32 words, L2[5])."""
    n = len(L)
    nb = (n + 127) // 128
    nw = (n + 15) // 16
    Lp = np.zeros(nb * 128, dtype=np.uint8)
    Lp[:n] = L
    valid = np.zeros(nb * 128, dtype=bool)
    valid[:n] = True
    blk = np.zeros((nb, 16), dtype=np.uint32)
    sym = Lp.reshape(nb * 8, 16).astype(np.uint32)
    shifts = (30 - 2 * np.arange(16)).astype(np.uint32)
    words = np.bitwise_or.reduce(sym << shifts[None, :], axis=1).reshape(nb, 8)
    blk[:, 8:] = words
    counts = np.zeros((nb, 4), dtype=np.uint64)
    for c in range(4):
        counts[:, c] = ((Lp == c) & valid).reshape(nb, 128).sum(axis=1)
    totals = counts.sum(axis=0)
    before = np.cumsum(counts, axis=0) - counts
    blk[:, :8] = before.astype(np.uint64).view(np.uint32).reshape(nb, 8)
    flat = blk.reshape(-1)
    last_words = nw - 8 * (nb - 1) if nb else 0
    body = flat[:16 * nb - (8 - last_words)] if nb else flat[:0]
    tail = totals.astype(np.uint64).view(np.uint32)
    L2 = np.zeros(5, dtype=np.uint64)
    L2[1:] = np.cumsum(totals)
    return np.concatenate([body, tail]), L2


def build_index(fasta: str, prefix: str, device: str | None = None) -> dict:
    """Writes <prefix>.pac/.ann/.amb/.bwt/.sa for a FASTA file. Returns a small summary."""
    names, comments, seqs = read_fasta(fasta)
    F = write_pac_ann_amb(prefix, names, comments, seqs)
    T = np.concatenate([F, (3 - F[::-1]).astype(np.uint8)])
    n = len(T)
    SA = suffix_array(T, device)
    primary = int(np.nonzero(SA == 0)[0][0])
    prev = SA - 1
    prev[primary] = 0
    Lfull = T[prev]
    L = np.delete(Lfull, primary)
    body, L2 = pack_bwt(L)
    with open(prefix + ".bwt", "wb") as f:
        np.array([primary], dtype=np.uint64).tofile(f)
        L2[1:].astype(np.uint64).tofile(f)
        body.astype(np.uint32).tofile(f)
    n_samples = (n + 32) // 32 - 1
    samples = SA[32 * np.arange(1, n_samples + 1)] if n_samples > 0 else np.zeros(0, np.int64)
    with open(prefix + ".sa", "wb") as f:
        np.array([primary], dtype=np.uint64).tofile(f)
        L2[1:].astype(np.uint64).tofile(f)
        np.array([32, n], dtype=np.uint64).tofile(f)
        samples.astype(np.uint64).tofile(f)
    return dict(n=n, primary=primary, L2=[int(x) for x in L2], prefix=prefix)


def build_from_reference(ref, prefix: str, device: str | None = None) -> dict:
    """Index a synth.Reference directly (writes its FASTA next to the index as <prefix>.fa)."""
    from galn_b200 import synth
    fa = prefix + ".fa"
    synth.write_fasta(fa, ref)
    return build_index(fa, prefix, device)


if __name__ == "__main__":
    import sys
    print(build_index(sys.argv[1], sys.argv[2]))
    os.sys.exit(0)
