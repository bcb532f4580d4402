"""Host-side logic of the C ABI (no GPU needed): the library loads and exports every entry point of
include/galn_aln.h; option parsing, bwa_cal_maxdiff, the FASTQ reader and the .sai writer agree with the
oracle and with the reference's golden files."""
import ctypes as C
import gzip
import os
import re
import subprocess

import numpy as np
import pytest

import galn_b200
import oracle
from conftest import GOLDEN, ROOT, case_paths, golden_cases
from galn_b200 import api, build

CASES = golden_cases()


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()
    oracle.build()


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "galn_aln.h")).read()
    names = set(re.findall(r"\b(galn_[a-z0-9_]+)\s*\(", header))
    assert len(names) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", api.lib_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (galn_[a-z0-9_]+)", out))
    missing = names - exported
    assert not missing, missing
    api.lib()
    assert galn_b200.lib().galn_version().startswith(b"galn-b200")


ARGSETS = [
    [], ["-n", "0.01", "-l", "1024", "-o", "2"], ["-n", "6", "-o", "2", "-e", "6", "-k", "3", "-N"],
    ["-L", "-n", "3", "-e", "2", "-R", "5", "-dt", "16"], ["-e", "0"], ["-e", "-1"], ["-t", "0"],
    ["-M", "4", "-O", "9", "-E", "2", "-d", "5", "-i", "3", "-m", "100", "-k", "1", "-l", "20"],
    ["-q", "0"], ["-n", "5.", "-N", "-L"], ["-n", ".5"],
]


@pytest.mark.parametrize("args", ARGSETS)
def test_option_block_matches_oracle(args):
    o = galn_b200.parse_options(args)
    assert bytes(o) == oracle.opt_bytes(oracle.parse_aln_args(args))


def test_option_errors():
    for bad in (["-q", "2"], ["-x", "1"], ["-n"]):
        with pytest.raises(galn_b200.GalnError):
            galn_b200.parse_options(bad)


def test_option_block_in_golden_sai(manifest):
    for name, meta in manifest.items():
        sai = open(case_paths(name, meta)["sai"], "rb").read()
        assert bytes(galn_b200.parse_options(meta["opts"])) == sai[4:68], name


def test_cal_maxdiff_matches_oracle():
    for thres in (np.float32(0.04), np.float32(0.01), np.float32(0.001), 0.5):
        for L in range(0, 400):
            assert galn_b200.cal_maxdiff(L, 0.02, float(thres)) == oracle.cal_maxdiff(L, 0.02, float(thres)), (L, thres)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fastq_reader_matches_oracle(name):
    p = case_paths(name, CASES[name])
    mine = galn_b200.read_fastq(p["fq"])
    ref = oracle.load_reads(p["fq"])
    np.testing.assert_array_equal(mine.offset, ref["off"])
    np.testing.assert_array_equal(mine.batch, ref["batch"])
    q = oracle.encode_queries(mine.seq, mine.offset)
    np.testing.assert_array_equal(q, ref["query"])


READER_EDGE = [
    b"@a\nACGT\n+\nIIII\n@b desc\nAC\r\nGT\r\n+\r\nII\r\nII\r\n",
    b"junk line\n>f1\nACGTN\nacgt\n>f2 c\n\n>f3\nA\n",
    b"@q1\nAAAA\n+\nII\n@q2\nCCCC\n+\nIIII\n@q3\nGG\n+\n",
    b"@e\n\n+\n\n@x\nT\n+\nI\n",
    b"@p\nAC-GT\n+\nIIIII\n@n\nNNNN\n+\n@@@@\n",
    b"@r\r\nACGT\r\n+\r\nIIII\r\n",
    b"@t\n\r\nAC\n+\nII",
    b"@u\nACGT\n+",
    b"",
    b"@v\nACGTACGT\n+\nIIII\nIIII\n@w\nA\n+\nI\n",
]


@pytest.mark.parametrize("i", range(len(READER_EDGE)))
def test_fastq_reader_edge_cases(i, tmp_path):
    path = str(tmp_path / f"e{i}.fq")
    with open(path, "wb") as f:
        f.write(READER_EDGE[i])
    mine = galn_b200.read_fastq(path)
    ref = oracle.load_reads(path)
    np.testing.assert_array_equal(mine.offset, ref["off"])
    np.testing.assert_array_equal(mine.batch, ref["batch"])
    np.testing.assert_array_equal(oracle.encode_queries(mine.seq, mine.offset), ref["query"])
    gz = path + ".gz"
    with gzip.open(gz, "wb") as f:
        f.write(READER_EDGE[i])
    mine2 = galn_b200.read_fastq(gz)
    np.testing.assert_array_equal(mine2.seq, mine.seq)


def _big_fastq(path, n, malformed_at=None):
    rng = np.random.default_rng(5)
    with open(path, "w") as f:
        for i in range(n):
            L = int(rng.integers(1, 40))
            s = "".join("ACGTN"[int(x)] for x in rng.integers(0, 5, L))
            if i == malformed_at:
                f.write(f"@bad{i}\n{s}A\n+\n{'I' * (L + 3)}\n")
            else:
                f.write(f"@r{i}\n{s}\n+\n{'I' * L}\n")


@pytest.mark.parametrize("case", list(range(len(READER_EDGE))) + ["big", "big_malformed"])
def test_fastq_batches_equal_whole_read(case, tmp_path):
    """Reading one bwa batch at a time gives the whole-file read's reads and batch ids, batch by batch
    (0x40000 reads per batch; a malformed record ends its batch)."""
    path = str(tmp_path / "b.fq")
    if case == "big":
        _big_fastq(path, 0x40000 + 1000)
    elif case == "big_malformed":
        _big_fastq(path, 0x40000 + 5000, malformed_at=1234)
    else:
        with open(path, "wb") as f:
            f.write(READER_EDGE[case])
    whole = galn_b200.read_fastq(path)
    parts = list(galn_b200.read_fastq_batches(path))
    n = sum(len(p) for p in parts)
    assert n == len(whole)
    if n:
        np.testing.assert_array_equal(np.concatenate([p.batch for p in parts]), whole.batch)
        seq = np.concatenate([p.seq for p in parts])
        np.testing.assert_array_equal(seq, whole.seq)
        lens = np.concatenate([np.diff(p.offset) for p in parts])
        np.testing.assert_array_equal(lens, np.diff(whole.offset))
        for p in parts:
            assert len(set(p.batch.tolist())) == 1
    if case == "big":
        assert [len(p) for p in parts] == [0x40000, 1000]
    if case == "big_malformed":
        assert len(parts) == 3 and len(parts[0]) < 0x40000


def test_fastq_reader_against_reference_harness(tmp_path):
    """The reference's own reader (read_fastq via the dump harness) on the reader edge cases."""
    if not oracle.ref_available():
        pytest.skip("reference binaries not built here")
    ob = oracle.opt_bytes(oracle.parse_aln_args([]))
    for i, data in enumerate(READER_EDGE):
        if not data:
            continue
        path = str(tmp_path / f"r{i}.fq")
        with open(path, "wb") as f:
            f.write(data)
        d = oracle.ref_dump(os.path.join(GOLDEN, "small", "ref.bwt"), path, ob, str(tmp_path / "d.bin"), 1)
        mine = galn_b200.read_fastq(path)
        np.testing.assert_array_equal(np.diff(mine.offset), d["len"])
        np.testing.assert_array_equal(mine.batch, d["batch"])


def test_sai_writer_matches_golden(tmp_path):
    """galn_sai_write over results taken from the golden .sai reproduces the file byte for byte."""
    for name, meta in CASES.items():
        p = case_paths(name, meta)
        sai = oracle.read_sai(p["sai"])
        n = len(sai["n_aln"])
        n_aln = np.ascontiguousarray(sai["n_aln"], np.int32)
        rec_off = np.zeros(n + 1, np.int64)
        rec_off[1:] = np.cumsum(np.maximum(n_aln, 0))
        recs = np.ascontiguousarray(sai["records"]) if len(sai["records"]) else np.zeros(1, api.REC_DTYPE)
        zeros = np.zeros(max(n, 1), np.uint64)
        r = api._Results()
        r.n_reads = n
        r.n_aln = n_aln.ctypes.data_as(C.POINTER(C.c_int32))
        r.rec_offset = rec_off.ctypes.data_as(C.POINTER(C.c_int64))
        r.rec = recs.ctypes.data
        r.n_pops = zeros.ctypes.data_as(C.POINTER(C.c_uint64))
        r.trace = zeros.ctypes.data_as(C.POINTER(C.c_uint64))
        o = galn_b200.parse_options(meta["opts"])
        out = str(tmp_path / (name + ".sai"))
        rc = galn_b200.lib().galn_sai_write(out.encode(), C.byref(o), C.byref(r))
        assert rc == 0
        assert open(out, "rb").read() == open(p["sai"], "rb").read(), name


def test_index_open_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(galn_b200.GalnError):
        galn_b200.Index(os.path.join(GOLDEN, "small", "ref"))


def test_cli_usage_and_errors(tmp_path):
    cli = build.CLI
    p = subprocess.run([cli], capture_output=True, text=True)
    assert p.returncode == 1 and "galn aln" in p.stderr
    p = subprocess.run([cli, "aln", "-q", "3", "a", "b"], capture_output=True, text=True)
    assert p.returncode == 1
    p = subprocess.run([cli, "aln", "--cpu-only", "a", "b"], capture_output=True, text=True)
    assert p.returncode == 1


@pytest.mark.parametrize("malformed", [None, 1234])
def test_gzip_input_read_ahead(malformed, tmp_path):
    """A gzip input is inflated ahead in a thread of its own: the whole-file and batch readers give the same
    reads as from the plain file, over several 8 MiB blocks and a batch boundary."""
    path = str(tmp_path / "b.fq")
    _big_fastq(path, 0x40000 + 3000, malformed_at=malformed)
    gz = path + ".gz"
    with open(path, "rb") as f, gzip.open(gz, "wb", compresslevel=1) as g:
        g.write(f.read())
    plain = galn_b200.read_fastq(path)
    whole = galn_b200.read_fastq(gz)
    np.testing.assert_array_equal(whole.seq, plain.seq)
    np.testing.assert_array_equal(whole.offset, plain.offset)
    np.testing.assert_array_equal(whole.batch, plain.batch)
    parts = list(galn_b200.read_fastq_batches(gz))
    np.testing.assert_array_equal(np.concatenate([p.seq for p in parts]), plain.seq)
    np.testing.assert_array_equal(np.concatenate([p.batch for p in parts]), plain.batch)


def test_gzip_input_closed_early_or_truncated(tmp_path):
    """Closing a gzip stream before its end stops the read-ahead; a truncated gzip file is an I/O error."""
    import ctypes as C
    path = str(tmp_path / "b.fq")
    _big_fastq(path, 0x40000 + 3000)
    gz = path + ".gz"
    with open(path, "rb") as f, gzip.open(gz, "wb", compresslevel=1) as g:
        g.write(f.read())
    it = galn_b200.read_fastq_batches(gz)
    assert len(next(it)) == 0x40000
    it.close()
    L = galn_b200.lib()
    err = C.c_int(0)
    st = L.galn_fastq_open(gz.encode(), C.byref(err))
    assert st and L.galn_fastq_close(st) == 0
    data = open(gz, "rb").read()
    cut = str(tmp_path / "cut.fq.gz")
    with open(cut, "wb") as f:
        f.write(data[: len(data) // 2])
    with pytest.raises(galn_b200.GalnError):
        galn_b200.read_fastq(cut)
