"""galn_aln_run_noalloc, the search entry point for callers that may not allocate device memory (their
framework owns the GPU's memory, or they run under a fixed budget, or must not trigger cudaFree's device
synchronisation). It takes the caller's device buffers and keeps its scratch in a fixed array inside the
library. This file is collected last so that a failure here leaves every other test already run; it
passes alone in a fresh process and after the rest of the suite.

Checked through the C ABI: on two calls in a row its n_aln and records equal those of the regular entry
point (galn_aln_run_batch) for every read it finishes, exactly (integer results, no tolerance); reads it
cannot finish within its fixed per-thread stack report GALN_ERR_STACK; the second call changes nothing in
the device's free memory; on a stream of its own, with one record per read, reads with more hits report
GALN_ERR_ALN and a read longer than max_len reports GALN_EINVAL while the others still match; sizes past
its limits are refused with GALN_EINVAL."""
import ctypes as C
import os

import numpy as np
import pytest

import galn_b200
from conftest import GOLDEN, case_paths, golden_cases
from galn_b200 import api, build

pytestmark = pytest.mark.gpu
GALN_EINVAL, GALN_ERR_STACK, GALN_ERR_ALN = -20, -1, -2
REC_PER_READ = 32


@pytest.fixture(scope="module")
def lib():
    build.build()
    L = galn_b200.lib()
    L.galn_aln_run_noalloc.argtypes = [C.c_void_p, C.POINTER(api.Options), C.c_int32, C.c_int32, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    return L


def _run(L, ix, opts, seq_d, off_d, n, max_len, n_aln_d, rec_d, stream, rec_per_read=REC_PER_READ):
    return L.galn_aln_run_noalloc(ix.h, C.byref(opts), n, max_len, seq_d.data_ptr(), off_d.data_ptr(),
                                  n_aln_d.data_ptr(), rec_d.data_ptr(), rec_per_read, stream)


def _golden_subset(name):
    """The golden case's reads of at most 1024 bases as one bwa batch, and the regular entry point's results."""
    meta = golden_cases()[name]
    p = case_paths(name, meta)
    ix = galn_b200.Index(os.path.join(GOLDEN, meta["ref"], "ref"))
    reads = galn_b200.read_fastq(p["fq"])
    keep = np.diff(reads.offset) <= 1024            # the entry point takes reads up to 1024 bases
    seqs = [bytes(reads.seq[reads.offset[i]:reads.offset[i + 1]]) for i in np.nonzero(keep)[0]]
    sub = galn_b200.Reads.from_strings(seqs)
    sub.batch = np.zeros(len(seqs), np.int32)      # one bwa batch, as the entry point treats its reads
    return meta, ix, seqs, sub, galn_b200.aln(ix, meta["opts"], sub)


def _check_records(ref, got_rec, rows):
    for r in rows:
        k = int(ref.n_aln[r])
        want = ref.records[ref.rec_offset[r]:ref.rec_offset[r] + k]
        have = got_rec[r, :k].view(np.uint64)
        np.testing.assert_array_equal(have[:, 0], want["packed"])
        np.testing.assert_array_equal(have[:, 1], want["k"])
        np.testing.assert_array_equal(have[:, 2], want["l"])


@pytest.mark.parametrize("name", ["plain", "adna", "genome", "edge_seed"])
def test_noalloc_matches_regular_entry_point(lib, name):
    import torch
    meta, ix, _, sub, ref = _golden_subset(name)
    n = len(sub)
    max_len = int(np.diff(sub.offset).max())
    opts = galn_b200.parse_options(meta["opts"])
    dev = torch.device("cuda:0")
    seq_d = torch.from_numpy(sub.seq.copy()).to(dev)
    off_d = torch.from_numpy(sub.offset.copy()).to(dev)
    n_aln_d = torch.full((n,), -99, dtype=torch.int32, device=dev)
    rec_d = torch.zeros((n, REC_PER_READ, 3), dtype=torch.int64, device=dev)
    stream = torch.cuda.current_stream(dev)
    outs = []
    for call in range(2):
        n_aln_d.fill_(-99)
        rec_d.zero_()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = _run(lib, ix, opts, seq_d, off_d, n, max_len, n_aln_d, rec_d, stream.cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info(dev)[0] == free_before, "the call allocated device memory"
        outs.append((n_aln_d.cpu().numpy().copy(), rec_d.cpu().numpy().copy()))
    for got_n, got_rec in outs:
        done = got_n != GALN_ERR_STACK
        assert done.mean() > 0.8, "too few reads finished within the fixed stack"
        np.testing.assert_array_equal(got_n[done], ref.n_aln[done])
        _check_records(ref, got_rec, np.nonzero(done & (ref.n_aln > 0))[0])
    np.testing.assert_array_equal(outs[0][0], outs[1][0])


def test_noalloc_record_limit_long_read_own_stream(lib):
    """One record per read on a stream of the test's own: reads with two or more hits stop at GALN_ERR_ALN;
    a read one base longer than max_len gets GALN_EINVAL; every other read equals the regular entry point."""
    import torch
    meta, ix, seqs, sub, ref = _golden_subset("plain")
    max_len = int(np.diff(sub.offset).max())
    at = len(seqs) // 2
    longer = seqs[:at] + [seqs[0][:1] * (max_len + 1)] + seqs[at:]
    both = galn_b200.Reads.from_strings(longer)
    n = len(both)
    opts = galn_b200.parse_options(meta["opts"])
    dev = torch.device("cuda:0")
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):
        seq_d = torch.from_numpy(both.seq.copy()).to(dev)
        off_d = torch.from_numpy(both.offset.copy()).to(dev)
        n_aln_d = torch.full((n,), -99, dtype=torch.int32, device=dev)
        rec_d = torch.zeros((n, 1, 3), dtype=torch.int64, device=dev)
        rc = _run(lib, ix, opts, seq_d, off_d, n, max_len, n_aln_d, rec_d, stream.cuda_stream, rec_per_read=1)
        assert rc == 0
    stream.synchronize()
    got_n = n_aln_d.cpu().numpy()
    got_rec = rec_d.cpu().numpy()
    assert got_n[at] == GALN_EINVAL
    got_n = np.delete(got_n, at)
    got_rec = np.delete(got_rec, at, axis=0)
    done = got_n != GALN_ERR_STACK
    assert done.mean() > 0.8
    many = ref.n_aln > 1
    assert many.any(), "the case needs reads with several hits"
    np.testing.assert_array_equal(got_n[done & many], GALN_ERR_ALN)
    np.testing.assert_array_equal(got_n[done & ~many], ref.n_aln[done & ~many])
    _check_records(ref, got_rec, np.nonzero(done & ~many & (ref.n_aln > 0))[0])


def test_noalloc_refuses_sizes_past_its_limits(lib):
    import torch
    ix = galn_b200.Index(os.path.join(GOLDEN, "small", "ref"))
    opts = galn_b200.parse_options([])
    dev = torch.device("cuda:0")
    seq_d = torch.zeros(16, dtype=torch.uint8, device=dev)
    off_d = torch.zeros(2, dtype=torch.int64, device=dev)
    n_aln_d = torch.zeros(1, dtype=torch.int32, device=dev)
    rec_d = torch.zeros((1, REC_PER_READ, 3), dtype=torch.int64, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    assert _run(lib, ix, opts, seq_d, off_d, 1, 1025, n_aln_d, rec_d, s) == GALN_EINVAL
    assert _run(lib, ix, opts, seq_d, off_d, 0x40001, 100, n_aln_d, rec_d, s) == GALN_EINVAL
    assert lib.galn_aln_run_noalloc(ix.h, C.byref(opts), 1, 100, seq_d.data_ptr(), off_d.data_ptr(),
                                    n_aln_d.data_ptr(), rec_d.data_ptr(), 257, s) == GALN_EINVAL
