"""`galn index` on the CPU side: the oracle's restatement of the .bwt/.sa files against the reference
builder's own files (tests/golden/index, tests/golden/small, tests/golden/genome: the pin), the oracle's
suffix sort against a plain sort, and the library's host step (FASTA -> .pac/.ann/.amb) against the
reference's files for every golden FASTA (CRLF, lowercase, IUPAC codes, empty and '@' records, gzip)."""
import filecmp
import gzip
import os

import numpy as np
import pytest

import galn_b200
import oracle
from conftest import GOLDEN

INDEX_CASES = sorted(os.listdir(os.path.join(GOLDEN, "index")))
ALL = [("index", c) for c in INDEX_CASES] + [("", "small"), ("", "genome")]


def _dir(group, name):
    return os.path.join(GOLDEN, group, name) if group else os.path.join(GOLDEN, name)


def _fasta(d):
    return os.path.join(d, "ref.fa.gz") if os.path.exists(os.path.join(d, "ref.fa.gz")) else os.path.join(d, "ref.fa")


@pytest.fixture(scope="module", autouse=True)
def _built():
    oracle.build()


def _same(a, b):
    return filecmp.cmp(a, b, shallow=False)


@pytest.mark.parametrize("group,name", ALL)
def test_oracle_index_files_are_the_references(group, name, tmp_path):
    d = _dir(group, name)
    F = oracle.forward_from_pac(os.path.join(d, "ref.pac"))
    pre = str(tmp_path / "o")
    oracle.index_files(F, pre)
    for ext in ("bwt", "sa"):
        assert _same(pre + "." + ext, os.path.join(d, "ref." + ext)), ext


def test_oracle_suffix_array_is_a_plain_sort():
    rng = np.random.default_rng(5)
    for n in (1, 2, 3, 7, 64, 300):
        for kind in range(3):
            T = (rng.integers(0, 4, n) if kind == 0 else np.zeros(n, np.int64) if kind == 1
                 else np.tile([0, 1], n)[:n]).astype(np.uint8)
            want = [n] + sorted(range(n), key=lambda i: T[i:].tobytes())
            np.testing.assert_array_equal(oracle.suffix_array(T), np.array(want, dtype=np.uint64))


@pytest.mark.parametrize("group,name", ALL)
def test_host_step_files_are_the_references(group, name, tmp_path):
    d = _dir(group, name)
    pre = str(tmp_path / "h")
    l_pac = galn_b200.fasta_to_pac(_fasta(d), pre)
    assert l_pac == len(oracle.forward_from_pac(os.path.join(d, "ref.pac")))
    for ext in ("pac", "ann", "amb"):
        assert _same(pre + "." + ext, os.path.join(d, "ref." + ext)), ext


def test_host_step_refuses_fastq_and_empty_input(tmp_path):
    fq = tmp_path / "r.fq"
    fq.write_text("@r1\nACGT\n+\nIIII\n")
    with pytest.raises(galn_b200.GalnError):
        galn_b200.fasta_to_pac(str(fq), str(tmp_path / "a"))
    empty = tmp_path / "e.fa"
    empty.write_text(">e\n\n")
    with pytest.raises(galn_b200.GalnError):
        galn_b200.fasta_to_pac(str(empty), str(tmp_path / "b"))
    with pytest.raises(galn_b200.GalnError):
        galn_b200.fasta_to_pac(str(tmp_path / "missing.fa"), str(tmp_path / "c"))


def test_forward_from_pac_round_trip(tmp_path):
    rng = np.random.default_rng(9)
    for n in (1, 3, 4, 5, 8, 1001):
        seq = "".join("ACGT"[i] for i in rng.integers(0, 4, n))
        fa = tmp_path / f"s{n}.fa.gz"
        with gzip.open(fa, "wt") as f:
            f.write(f">s\n{seq}\n")
        galn_b200.fasta_to_pac(str(fa), str(tmp_path / f"s{n}"))
        F = oracle.forward_from_pac(str(tmp_path / f"s{n}.pac"))
        assert "".join("ACGT"[c] for c in F) == seq


def test_command_line_options_without_a_gpu(tmp_path):
    """`galn index` refuses the CPU builder, unknown builders and options, and a missing FASTA argument with
    exit code 1 before touching a device."""
    import subprocess
    from galn_b200 import build
    build.build()
    fa = os.path.join(GOLDEN, "index", "tiny3", "ref.fa")
    pre = ["-p", str(tmp_path / "x")]
    for args in (pre, pre + ["-a", "cpu", fa], pre + ["--cpu", fa], pre + ["-a", "bogus", fa], pre + ["--bogus", fa],
                 pre + [fa, fa]):
        p = subprocess.run([build.CLI, "index", *args], capture_output=True, text=True)
        assert p.returncode == 1, (args, p.stderr)
        assert not os.path.exists(str(tmp_path / "x.pac"))


def test_oracle_suffix_array_agrees_with_prefix_doubling():
    """The oracle's comparison sort and the fixture builder's prefix doubling (torch on the CPU) are two
    independent suffix sorts: they agree on random, repetitive and palindromic texts."""
    import fixture_index as index_build
    rng = np.random.default_rng(31)
    u = rng.integers(0, 4, 3000)
    for T in (rng.integers(0, 4, 40_000), np.tile(u[:37], 300), np.concatenate([u, 3 - u[::-1], u, u[:1000]])):
        T = T.astype(np.uint8)
        np.testing.assert_array_equal(oracle.suffix_array(T).astype(np.int64), index_build.suffix_array(T, "cpu"))


def test_host_step_random_fasta_against_fixture_writer(tmp_path):
    """Random FASTA files (records of random length, lowercase, runs of IUPAC codes, wrapped at random widths)
    give the same .pac/.ann/.amb from the library's host step as from the fixture builder's writer."""
    import fixture_index as index_build
    rng = np.random.default_rng(8)
    alphabet = np.frombuffer(b"ACGTACGTACGTacgtNNRYKMnSW", dtype=np.uint8)
    for case in range(12):
        parts = []
        for r in range(int(rng.integers(1, 8))):
            L = int(rng.integers(0 if r else 1, 3000))
            seq = alphabet[rng.integers(0, len(alphabet), L)]
            if L > 50:   # a long run of one ambiguous code
                a = int(rng.integers(0, L - 40))
                seq[a:a + 30] = ord("N")
            w = int(rng.integers(10, 120))
            body = b"".join(seq[i:i + w].tobytes() + b"\n" for i in range(0, L, w))
            head = b">c%d" % r + (b" some comment %d" % case if r % 2 else b"")
            parts.append(head + b"\n" + body)
        fa = tmp_path / f"r{case}.fa"
        fa.write_bytes(b"".join(parts))
        galn_b200.fasta_to_pac(str(fa), str(tmp_path / f"h{case}"))
        names, comments, seqs = index_build.read_fasta(str(fa))
        index_build.write_pac_ann_amb(str(tmp_path / f"f{case}"), names, comments, seqs)
        for ext in ("pac", "ann", "amb"):
            assert _same(str(tmp_path / f"h{case}.{ext}"), str(tmp_path / f"f{case}.{ext}")), (case, ext)


@pytest.mark.parametrize("n", [1, 15, 16, 17, 127, 128, 129, 255, 1000, 5077])
def test_random_bwt_helper_matches_brute_force(n, tmp_path):
    """The random .bwt files of the superblock test: the oracle's Occ over them equals a count over their
    symbols at every row, also when the file is assembled in several chunks."""
    import bwt_synth
    rng = np.random.default_rng(n)
    primary = int(rng.integers(1, n + 1))
    for chunk in (1 << 22, 3):
        words = bwt_synth.random_bwt(n, primary, seed=n, chunk_blocks=chunk)
        path = str(tmp_path / f"r{chunk}.bwt")
        words.tofile(path)
        sym = bwt_synth.symbols(words)
        rows = np.concatenate([np.arange(n + 1, dtype=np.uint64), np.array([(1 << 64) - 1], np.uint64)])
        got = oracle.Index(path).occ4(rows)
        np.testing.assert_array_equal(got, bwt_synth.occ_brute(sym, primary, rows))


def test_fixture_builder_from_reference(tmp_path):
    """The fixture builder indexes a synthetic reference directly (on the host here) with the oracle's
    .bwt and .sa."""
    import fixture_index
    from galn_b200 import synth
    ref = synth.reference_adna(20_000, 5, n_contigs=2)
    fixture_index.build_from_reference(ref, str(tmp_path / "fx"), "cpu")
    F = oracle.forward_from_pac(str(tmp_path / "fx.pac"))
    oracle.index_files(F, str(tmp_path / "o"))
    for ext in ("bwt", "sa"):
        assert filecmp.cmp(str(tmp_path / ("fx." + ext)), str(tmp_path / ("o." + ext)), shallow=False), ext
