"""Regenerates tests/golden/index/: FASTA inputs that exercise `galn index`'s record and base rules, and the
five files the reference's own CPU builder (oracle/_ref/galn_index_cpu, `galn index -a cpu`) writes for them.

Needs the reference sources (the oracle Makefile builds galn_index_cpu from them); run once where they are
present:

    python tests/golden/make_index_golden.py

Cases: CRLF line ends with lowercase bases and odd headers; IUPAC codes and runs of ambiguous bases at
record edges; many short records with an empty one, an '@' header and text before the first '>'; a
reference whose length is a multiple of 4 made of a homopolymer and tandem repeats; 1- and 3-base
references; long exact and reverse-complement repeats (many doubling rounds); a gzip input.
"""
from __future__ import annotations

import gzip
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

OUT = os.path.join(HERE, "index")


def rand_bases(rng, n, alphabet=b"ACGT"):
    a = np.frombuffer(alphabet, dtype=np.uint8)
    return a[rng.integers(0, len(a), n)].tobytes()


def wrap(seq: bytes, width=60, eol=b"\n") -> bytes:
    return b"".join(seq[i:i + width] + eol for i in range(0, len(seq), width))


def cases():
    rng = np.random.default_rng(2024)
    out = {}
    # CRLF, lowercase, a tab and double spaces in headers, a name-only header, a "\r" line first
    s1 = rand_bases(rng, 700, b"ACGTacgt")
    s2 = rand_bases(rng, 333)
    out["crlf"] = (b">chr1 first\tcontig  with spaces\r\n" + wrap(s1, 70, b"\r\n") +
                   b">chr2\r\n" + wrap(s2, 50, b"\r\n") +
                   b">chr3 x\r\n\r\n" + wrap(rand_bases(rng, 90), 45, b"\r\n") +
                   b">chr4 \r\n" + wrap(rand_bases(rng, 17), 60, b"\r\n"))
    # IUPAC codes, ambiguous runs at record starts and ends, alternating different ambiguous bases
    body = bytearray(rand_bases(rng, 1500))
    for p, run in ((0, b"NNNN"), (100, b"RYRYRY"), (400, b"nnnnNNNN"), (700, b"K"), (1496, b"MMMM")):
        body[p:p + len(run)] = run
    out["iupac"] = (b">amb1 ambiguous bases\n" + wrap(bytes(body)) +
                    b">amb2\n" + wrap(b"NNN" + rand_bases(rng, 200) + b"SSWW" + rand_bases(rng, 5) + b"N") +
                    b">amb3\n" + wrap(b"ACGTBDHVN.-*acgtu"))
    # many short records, an empty one, an '@' header, text before the first '>'
    parts = [b"stray text before the first record\n"]
    for i in range(40):
        L = int(rng.integers(1, 30))
        parts.append(b">r%d\n" % i + wrap(rand_bases(rng, L)))
        if i == 7:
            parts.append(b">empty record\n")
        if i == 20:
            parts.append(b"@at_header\n" + wrap(rand_bases(rng, 12)))
    out["contigs"] = b"".join(parts)
    # length a multiple of 4: homopolymer and tandem repeats
    seq = b"A" * 1500 + b"ACGT" * 300 + b"CAG" * 200 + rand_bases(rng, 196)
    assert len(seq) % 4 == 0
    out["lpac4"] = b">rep\n" + wrap(seq)
    out["tiny1"] = b">one\nA\n"
    out["tiny3"] = b">three\nACG\n"
    # long exact and reverse-complement repeats
    u = rand_bases(rng, 3000)
    rc = u[::-1].translate(bytes.maketrans(b"ACGT", b"TGCA"))
    seq = rand_bases(rng, 500) + u + rand_bases(rng, 200) + u + u[:1700] + rc + rand_bases(rng, 300)
    out["repeats"] = b">r1\n" + wrap(seq) + b">r2\n" + wrap(u[1000:2500])
    return out


def main():
    oracle.build(ref=True)
    if os.path.isdir(OUT):
        shutil.rmtree(OUT)
    for name, data in cases().items():
        d = os.path.join(OUT, name)
        os.makedirs(d)
        fa = os.path.join(d, "ref.fa")
        with open(fa, "wb") as f:
            f.write(data)
        subprocess.run([oracle.INDEX_REF, "-f", fa, os.path.join(d, "ref")], check=True, capture_output=True)
    # the gzip input: the repeats case compressed, same index files
    d = os.path.join(OUT, "gz")
    os.makedirs(d)
    with open(os.path.join(OUT, "repeats", "ref.fa"), "rb") as f, gzip.open(os.path.join(d, "ref.fa.gz"), "wb") as g:
        g.write(f.read())
    subprocess.run([oracle.INDEX_REF, "-f", os.path.join(d, "ref.fa.gz"), os.path.join(d, "ref")], check=True,
                   capture_output=True)
    for name in sorted(os.listdir(OUT)):
        print(name, sorted(os.listdir(os.path.join(OUT, name))))


if __name__ == "__main__":
    main()
