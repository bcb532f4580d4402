"""Seeded synthetic references and reads with the shapes of the aln workloads.

The reference's published runs use ENA read sets and large genomes that are not available here; these
generators stand in for them with the same shapes: read-length distributions, error and deamination
profiles, repeat content and reference sizes. Everything is drawn from numpy's PCG64 with a fixed seed, so
the same call gives the same bytes on every machine.

Workloads (names follow the read/reference shapes, sizes are the defaults):
  plain_small   1 Mbp uniform ACGT, 1 contig; 20,000 x 100 bp reads from both strands, 1% substitutions,
                0.1% indels of 1-3 bp, 2% fully random reads, Phred 20-40; default aln options.
  adna          100 Mbp at 45% GC in 10 contigs with 5% interspersed repeats (300 bp families, copies at
                10% divergence); 2 M reads, log-normal length (mean 50, 25-120 bp), 0.5% substitutions,
                5' C->T 30% at position 1 decaying x0.5 per base and mirrored 3' G->A, 3% random reads;
                options -l 1024 -n 0.01 -o 2.
  divergent     the adna reference; 1 M x 100 bp reads at 4% substitutions + 0.5% indels;
                options -n 6 -o 2 -e 6 -k 3 -N.
  genome        24 contigs from 250 down to 50 Mbp (3.1 Gbp at full size), 50% repeats (Alu-like 300 bp
                at 15% divergence, L1-like 6 kbp, 2-50 bp tandem repeats), 0.3% N runs; 150 bp reads with
                a substitution rate ramping 0.1% -> 1.5% along the read plus 0.05% indels; default options.
Every generator takes a `scale` so that tests can run the same shapes at a fraction of the size.
"""
from __future__ import annotations

import gzip
import math
import os
from dataclasses import dataclass, field

import numpy as np

ASCII = np.frombuffer(b"ACGTN", dtype=np.uint8)
COMP = np.array([3, 2, 1, 0, 4], dtype=np.uint8)

ADNA_OPTS = ["-l", "1024", "-n", "0.01", "-o", "2"]
DIVERGENT_OPTS = ["-n", "6", "-o", "2", "-e", "6", "-k", "3", "-N"]
DEFAULT_OPTS: list[str] = []


@dataclass
class Reference:
    names: list[str]
    seqs: list[np.ndarray]          # codes 0..3, 4 = N

    @property
    def total(self) -> int:
        return int(sum(len(s) for s in self.seqs))


@dataclass
class Reads:
    names: list[str]
    seq: np.ndarray                 # concatenated codes 0..4
    off: np.ndarray                 # int64 offsets, len n+1
    qual: np.ndarray | None = None  # concatenated Phred values
    meta: dict = field(default_factory=dict)

    def __len__(self) -> int:
        return len(self.off) - 1

    @property
    def lengths(self) -> np.ndarray:
        return np.diff(self.off).astype(np.int32)

    def ascii(self) -> np.ndarray:
        return ASCII[self.seq]


# ---------------------------------------------------------------------------------------------
# references

def _random_bases(rng: np.random.Generator, n: int, gc: float = 0.5) -> np.ndarray:
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    return rng.choice(4, size=n, p=p).astype(np.uint8)


def _mutate(rng: np.random.Generator, s: np.ndarray, rate: float) -> np.ndarray:
    s = s.copy()
    m = rng.random(len(s)) < rate
    s[m] = (s[m] + rng.integers(1, 4, size=int(m.sum()), dtype=np.uint8)) % 4
    return s


def _insert_copies(rng, seq: np.ndarray, family: np.ndarray, n_copies: int, divergence: float) -> None:
    L = len(family)
    if len(seq) <= L:
        return
    pos = rng.integers(0, len(seq) - L, size=n_copies)
    for p in pos:
        c = _mutate(rng, family, divergence)
        if rng.random() < 0.5:
            c = COMP[c[::-1]]
        seq[p:p + L] = c


def reference_uniform(total: int, seed: int, n_contigs: int = 1) -> Reference:
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = [total // n_contigs] * n_contigs
    sizes[-1] += total - sum(sizes)
    return Reference([f"chr{i + 1}" for i in range(n_contigs)], [_random_bases(rng, s) for s in sizes])


def reference_adna(total: int, seed: int, n_contigs: int = 10, gc: float = 0.45,
                   repeat_frac: float = 0.05, family_len: int = 300, n_families: int = 50,
                   divergence: float = 0.10) -> Reference:
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = [total // n_contigs] * n_contigs
    sizes[-1] += total - sum(sizes)
    seqs = [_random_bases(rng, s, gc) for s in sizes]
    fams = [_random_bases(rng, family_len, gc) for _ in range(n_families)]
    n_copies = int(repeat_frac * total / family_len)
    owner = rng.integers(0, n_contigs, size=n_copies)
    fam_of = rng.integers(0, n_families, size=n_copies)
    for ci in range(n_contigs):
        sel = fam_of[owner == ci]
        for f in range(n_families):
            k = int((sel == f).sum())
            if k:
                _insert_copies(rng, seqs[ci], fams[f], k, divergence)
    return Reference([f"chr{i + 1}" for i in range(n_contigs)], seqs)


def _genome_sizes(total: int, n: int = 24, big: float = 250e6, small: float = 50e6, full: float = 3.1e9):
    """Contig sizes falling from `big` to `small` on a power curve whose sum is `full`, scaled to `total`."""
    x = np.linspace(1.0, 0.0, n)
    lo, hi = 0.01, 20.0
    for _ in range(100):
        p = (lo + hi) / 2
        s = (small + (big - small) * x ** p).sum()
        lo, hi = (p, hi) if s > full else (lo, p)
    sizes = small + (big - small) * x ** p
    sizes = np.maximum(1, np.round(sizes * total / sizes.sum())).astype(np.int64)
    sizes[0] += total - sizes.sum()
    return [int(v) for v in sizes]


def reference_genome(total: int, seed: int, n_contigs: int = 24, n_frac: float = 0.003) -> Reference:
    rng = np.random.Generator(np.random.PCG64(seed))
    sizes = _genome_sizes(total, n_contigs)
    seqs = [_random_bases(rng, s, 0.41) for s in sizes]
    alu = [_random_bases(rng, 300, 0.52) for _ in range(20)]
    l1 = [_random_bases(rng, 6000, 0.40) for _ in range(5)]
    # 50% repeats: 20% Alu-like, 25% L1-like, 5% tandem
    for ci, s in enumerate(seqs):
        L = len(s)
        n_alu = int(0.20 * L / 300)
        for f, k in zip(*np.unique(rng.integers(0, len(alu), size=n_alu), return_counts=True)):
            _insert_copies(rng, s, alu[f], int(k), 0.15)
        n_l1 = int(0.25 * L / 6000)
        for f, k in zip(*np.unique(rng.integers(0, len(l1), size=n_l1), return_counts=True)):
            _insert_copies(rng, s, l1[f], int(k), 0.08)
        tandem_bases = int(0.05 * L)
        done = 0
        while done < tandem_bases and L > 200:
            unit = _random_bases(rng, int(rng.integers(2, 51)))
            copies = int(rng.integers(3, 40))
            block = np.tile(unit, copies)
            block = _mutate(rng, block, 0.02)
            p = int(rng.integers(0, max(1, L - len(block))))
            s[p:p + len(block)] = block[:L - p]
            done += len(block)
        n_bases = int(n_frac * L)
        done = 0
        while done < n_bases and L > 2000:
            run = int(rng.integers(50, 1000))
            p = int(rng.integers(0, L - run))
            s[p:p + run] = 4
            done += run
    return Reference([f"chr{i + 1}" for i in range(n_contigs)], seqs)


def write_fasta(path: str, ref: Reference, width: int = 60) -> None:
    with open(path, "wb") as f:
        for name, s in zip(ref.names, ref.seqs):
            f.write(b">" + name.encode() + b"\n")
            a = ASCII[s]
            n = len(a)
            full = n // width
            if full:
                block = np.empty((full, width + 1), dtype=np.uint8)
                block[:, :width] = a[:full * width].reshape(full, width)
                block[:, width] = 10
                f.write(block.tobytes())
            if n % width:
                f.write(a[full * width:].tobytes() + b"\n")


# ---------------------------------------------------------------------------------------------
# reads

def _sample_positions(rng, ref: Reference, lens: np.ndarray):
    """Start positions (global offset in the concatenated reference) fully inside one contig."""
    sizes = np.array([len(s) for s in ref.seqs], dtype=np.int64)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    n = len(lens)
    ci = rng.choice(len(sizes), size=n, p=sizes / sizes.sum())
    room = np.maximum(1, sizes[ci] - 2 * lens.astype(np.int64) - 8)
    return starts[ci] + (rng.random(n) * room).astype(np.int64)


def _simulate(rng, flat: np.ndarray, pos: np.ndarray, lens: np.ndarray, sub_rate, indel_rate: float,
              random_frac: float, deaminate: float = 0.0) -> tuple[np.ndarray, np.ndarray]:
    """Reads of the given lengths as (concatenated codes, offsets). sub_rate: scalar or a function of the
    relative position in the read (0..1). Indels 1-3 bp, insertions and deletions equally likely."""
    n = len(lens)
    Lmax = int(lens.max()) if n else 0
    W = 2 * Lmax + 16
    j = np.arange(Lmax)[None, :]
    valid = j < lens[:, None]
    # indel events per output position
    ev = rng.random((n, Lmax))
    is_ins = (ev < indel_rate / 2) & valid
    is_del = (ev >= indel_rate / 2) & (ev < indel_rate) & valid
    ilen = rng.integers(1, 4, size=(n, Lmax))
    del_len = np.where(is_del, ilen, 0)
    consume = np.where(is_ins, 0, 1 + del_len)
    src = np.cumsum(consume, axis=1) - consume + del_len
    src = np.minimum(src, W - 1)
    win = flat[pos[:, None] + np.arange(W)[None, :]]
    out = np.take_along_axis(win, src, axis=1)
    out = np.where(is_ins, rng.integers(0, 4, size=(n, Lmax)).astype(np.uint8), out)
    # strand: reverse-complement half of the reads (within their own length)
    rev = rng.random(n) < 0.5
    if rev.any():
        r = out[rev]
        lr = lens[rev]
        idx = (lr[:, None] - 1 - j) % Lmax
        idx = np.where(j < lr[:, None], idx, j)
        r = np.take_along_axis(r, idx, axis=1)
        out[rev] = np.where(j < lr[:, None], COMP[r], r)
    # substitutions
    if callable(sub_rate):
        rate = sub_rate(j / np.maximum(1, lens[:, None] - 1))
    else:
        rate = np.full((1, Lmax), float(sub_rate))
    sub = (rng.random((n, Lmax)) < rate) & valid & (out < 4)
    out = np.where(sub, (out + rng.integers(1, 4, size=(n, Lmax))) % 4, out).astype(np.uint8)
    # deamination: C->T at the 5' end, G->A at the 3' end of the sequenced molecule
    if deaminate > 0:
        p5 = deaminate * 0.5 ** j
        p3 = deaminate * 0.5 ** (lens[:, None] - 1 - j)
        u = rng.random((n, Lmax))
        out = np.where((out == 1) & (u < p5) & valid, 3, out)
        u = rng.random((n, Lmax))
        out = np.where((out == 2) & (u < p3) & valid, 0, out).astype(np.uint8)
    # fully random reads
    rnd = rng.random(n) < random_frac
    if rnd.any():
        out[rnd] = rng.integers(0, 4, size=(int(rnd.sum()), Lmax)).astype(np.uint8)
    seq = out[valid]
    off = np.concatenate([[0], np.cumsum(lens.astype(np.int64))])
    return seq, off


def simulate_reads(ref: Reference, n: int, seed: int, length, sub_rate=0.01, indel_rate=0.0,
                   random_frac=0.0, deaminate: float = 0.0, prefix: str = "r", chunk: int = 1 << 17) -> Reads:
    """`length`: an int, or a callable rng, n -> int array of lengths."""
    rng = np.random.Generator(np.random.PCG64(seed))
    flat = np.concatenate(ref.seqs + [np.full(4096, 4, dtype=np.uint8)])
    seqs, offs = [], []
    base = 0
    for c0 in range(0, n, chunk):
        m = min(chunk, n - c0)
        lens = (np.full(m, int(length), dtype=np.int32) if not callable(length)
                else np.asarray(length(rng, m), dtype=np.int32))
        pos = _sample_positions(rng, ref, lens)
        s, o = _simulate(rng, flat, pos, lens, sub_rate, indel_rate, random_frac, deaminate)
        seqs.append(s)
        offs.append(o[:-1] + base)
        base += int(o[-1])
    seq = np.concatenate(seqs) if seqs else np.zeros(0, np.uint8)
    off = np.concatenate(offs + [np.array([base], dtype=np.int64)])
    qual = rng.integers(20, 41, size=len(seq)).astype(np.uint8)
    names = [f"{prefix}{i:08d}" for i in range(n)]
    return Reads(names, seq, off, qual)


def adna_lengths(rng, m):
    # log-normal with mean 50 (sigma 0.45 on the log scale), clipped to 25..120
    sigma = 0.45
    mu = math.log(50) - sigma * sigma / 2
    return np.clip(np.round(rng.lognormal(mu, sigma, size=m)), 25, 120).astype(np.int32)


def write_fastq(path: str, reads: Reads) -> None:
    opener = gzip.open if path.endswith(".gz") else open
    a = reads.ascii()
    q = (reads.qual + 33).astype(np.uint8) if reads.qual is not None else np.full(len(a), ord("I"), np.uint8)
    ab, qb = a.tobytes(), q.tobytes()
    off = reads.off
    with opener(path, "wb") as f:
        buf = []
        for i, name in enumerate(reads.names):
            s, e = int(off[i]), int(off[i + 1])
            buf.append(b"@%s\n%s\n+\n%s\n" % (name.encode(), ab[s:e], qb[s:e]))
            if len(buf) >= 65536:
                f.write(b"".join(buf))
                buf = []
        f.write(b"".join(buf))


# ---------------------------------------------------------------------------------------------
# the named workloads

FULL_READS = {"plain_small": 20_000, "adna": 2_000_000, "divergent": 1_000_000, "genome": 10_000_000}


def workload_reference(name: str, scale: float = 1.0, seed: int = 1) -> Reference:
    """The reference of a named workload at `scale` of its full size (divergent shares adna's)."""
    if name == "plain_small":
        return reference_uniform(max(10_000, int(1_000_000 * scale)), seed)
    if name in ("adna", "divergent"):
        return reference_adna(max(20_000, int(100_000_000 * scale)), seed)
    if name == "genome":
        return reference_genome(max(200_000, int(3_100_000_000 * scale)), seed)
    raise KeyError(name)


def workload_reads(name: str, ref: Reference, n: int, seed: int = 1) -> tuple[Reads, list[str]]:
    """n reads of a named workload drawn from `ref` (the reads workload() returns for the same seed), and
    the workload's aln options."""
    if name == "plain_small":
        return (simulate_reads(ref, n, seed + 1, 100, sub_rate=0.01, indel_rate=0.001, random_frac=0.02,
                               prefix="ps"), list(DEFAULT_OPTS))
    if name == "adna":
        return (simulate_reads(ref, n, seed + 1, adna_lengths, sub_rate=0.005, random_frac=0.03, deaminate=0.3,
                               prefix="ad"), list(ADNA_OPTS))
    if name == "divergent":
        return (simulate_reads(ref, n, seed + 2, 100, sub_rate=0.04, indel_rate=0.005, prefix="dv"),
                list(DIVERGENT_OPTS))
    if name == "genome":
        return (simulate_reads(ref, n, seed + 3, 150, sub_rate=lambda x: 0.001 + 0.014 * x, indel_rate=0.0005,
                               prefix="gn"), list(DEFAULT_OPTS))
    raise KeyError(name)


def workload(name: str, scale: float = 1.0, seed: int = 1, reads_scale: float | None = None):
    """(reference, reads, options) for a named workload at `scale` of its full size (the reads at
    `reads_scale` of theirs when given)."""
    rs = scale if reads_scale is None else reads_scale
    ref = workload_reference(name, scale, seed)
    reads, opts = workload_reads(name, ref, max(1, int(FULL_READS[name] * rs)), seed)
    return ref, reads, opts


def serving_requests(n_requests: int, seed: int, ref: Reference, scale: float = 1.0,
                     min_reads: int = 1000, max_reads: int = 500_000, rate_hz: float = 20.0):
    """Request stream for the serving workload: Poisson arrivals, request sizes log-uniform in
    [min_reads, max_reads] (times `scale`), read lengths 36-150 bp, half default and half aDNA options.
    Returns a list of dicts {t_arrival, reads, opts}."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    lo, hi = math.log(max(1, min_reads * scale)), math.log(max(2, max_reads * scale))
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate_hz)
        n = int(round(math.exp(rng.uniform(lo, hi))))
        adna = bool(i % 2)
        reads = simulate_reads(ref, n, seed * 1000 + i, lambda r, m: r.integers(36, 151, size=m),
                               sub_rate=0.005 if adna else 0.01, random_frac=0.03,
                               deaminate=0.3 if adna else 0.0, prefix=f"q{i}_")
        out.append(dict(t_arrival=t, reads=reads, opts=list(ADNA_OPTS if adna else DEFAULT_OPTS)))
    return out


def write_workload(dirpath: str, name: str, scale: float = 1.0, seed: int = 1, gz: bool = False):
    os.makedirs(dirpath, exist_ok=True)
    ref, reads, opts = workload(name, scale, seed)
    fa = os.path.join(dirpath, "ref.fa")
    fq = os.path.join(dirpath, "reads.fq" + (".gz" if gz else ""))
    write_fasta(fa, ref)
    write_fastq(fq, reads)
    return fa, fq, opts
