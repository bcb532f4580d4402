"""Test infrastructure: the CPU oracle for the `bwa aln` search, and the reference itself.

Only tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs of bench.py use this package,
and only as the checker (or, for the reference legs, as the timed CPU baseline and the reference arm's index
builder); the product never imports it.

  * liboracle.so          this project's own C restatement of the reference's search, of bwt_sa/bwa_sa2pos and
                          of the .bwt/.sa index files over a comparison suffix sort (galn_oracle.c)
  * _ref/galn_ref         the reference's `galn aln` built from its own sources (oracle/Makefile)
  * _ref/galn_index_cpu   the reference's CPU index builder
  * _ref/libgalnref_dump.so  per-read dump around the reference's aln_search_host

`parse_aln_args` restates the reference's option parsing (galn.cu:185-250 with the defaults of
opt_build.h:23-36) to build the 64-byte option block written into the .sai header.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")
LIB_PATH = os.path.join(BUILD, "liboracle.so")
GALN_REF = os.path.join(REF, "galn_ref")
INDEX_REF = os.path.join(REF, "galn_index_cpu")
DUMP_REF = os.path.join(REF, "libgalnref_dump.so")

OPT_FMT = "<7if8i"          # gap_opt_t: 7 ints, float fnr, 8 ints = 64 bytes
REC_DTYPE = np.dtype([("packed", "<u8"), ("k", "<u8"), ("l", "<u8")])
MODE_GAPE, MODE_COMPREAD, MODE_LOGGAP, MODE_NONSTOP = 0x01, 0x02, 0x04, 0x10


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and, with ref=True and the reference sources present, the _ref binaries)."""
    target = ["oracle"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + target, check=True)


def reference_sources_present() -> bool:
    """Whether the reference's sources are where oracle/Makefile looks for them (GALN_REFERENCE)."""
    p = subprocess.run(["make", "-s", "-C", HERE, "ref-present"], capture_output=True)
    return p.returncode == 0


def ref_available() -> bool:
    return os.path.exists(GALN_REF) and os.path.exists(DUMP_REF)


# ------------------------------------------------------------------------------------------------
# options (galn.cu:185-250)

def default_opts() -> dict:
    return dict(s_mm=3, s_gapo=11, s_gape=4, mode=MODE_GAPE | MODE_COMPREAD, indel_end_skip=5,
                max_del_occ=10, max_entries=2000000, fnr=0.04, max_diff=-1, max_gapo=1, max_gape=6,
                max_seed_diff=2, seed_len=32, n_threads=1, max_top2=30, trim_qual=0)


def parse_aln_args(args: list[str]) -> dict:
    """The option block the reference writes for `galn aln <args>` (without positional arguments)."""
    o = default_opts()
    opte = -1
    i = 0
    while i < len(args):
        a = args[i]
        if a == "-L":
            o["mode"] |= MODE_LOGGAP
        elif a == "-N":
            o["mode"] |= MODE_NONSTOP
            o["max_top2"] = 0x7FFFFFFF
        else:
            v = args[i + 1]
            i += 1
            if a == "-n":
                if "." in v:
                    o["fnr"], o["max_diff"] = float(v), -1
                else:
                    o["max_diff"], o["fnr"] = int(v), -1.0
            elif a == "-e":
                opte = int(v)
            elif a == "-q":
                if int(v) >= 1:
                    raise ValueError("-q (quality trimming) is not supported")
            elif a == "-f":
                pass
            else:
                key = {"-o": "max_gapo", "-M": "s_mm", "-O": "s_gapo", "-E": "s_gape", "-d": "max_del_occ",
                       "-i": "indel_end_skip", "-l": "seed_len", "-k": "max_seed_diff", "-m": "max_entries",
                       "-dt": "n_threads", "-t": "n_threads", "-R": "max_top2"}[a]
                o[key] = int(v)
        i += 1
    if opte > 0:
        o["max_gape"] = opte
        o["mode"] &= ~MODE_GAPE
    if o["n_threads"] < 1:
        o["n_threads"] = 1
    return o


def opt_bytes(o: dict) -> bytes:
    return struct.pack(OPT_FMT, o["s_mm"], o["s_gapo"], o["s_gape"], o["mode"], o["indel_end_skip"],
                       o["max_del_occ"], o["max_entries"], o["fnr"], o["max_diff"], o["max_gapo"], o["max_gape"],
                       o["max_seed_diff"], o["seed_len"], o["n_threads"], o["max_top2"], o["trim_qual"])


# ------------------------------------------------------------------------------------------------
# liboracle

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, ip, i64p = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int64)
        L.orc_index_load.restype = vp
        L.orc_index_load.argtypes = [C.c_char_p, ip]
        L.orc_index_free.argtypes = [vp]
        L.orc_index_meta.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.orc_occ4.argtypes = [vp, vp, C.c_int64, vp]
        L.orc_index_borrow.restype = vp
        L.orc_index_borrow.argtypes = [vp, C.c_uint64, ip]
        L.orc_reads_load.restype = vp
        L.orc_reads_load.argtypes = [C.c_char_p, ip, i64p, ip]
        L.orc_reads_get.argtypes = [vp, vp, vp, vp, vp]
        L.orc_reads_free.argtypes = [vp]
        L.orc_cal_maxdiff.argtypes = [C.c_int, C.c_double, C.c_double]
        L.orc_aln.restype = vp
        L.orc_aln.argtypes = [vp, C.c_char_p, vp, vp, vp, vp, C.c_int, C.c_int]
        L.orc_aln_bmax.restype = vp
        L.orc_aln_bmax.argtypes = [vp, C.c_char_p, vp, vp, vp, vp, C.c_int, C.c_int, vp, C.c_int]
        L.orc_result_total.restype = C.c_int64
        L.orc_result_total.argtypes = [vp]
        L.orc_result_dump.argtypes = [vp] + [vp] * 10
        L.orc_result_write_sai.argtypes = [vp, C.c_char_p, C.c_char_p]
        L.orc_result_free.argtypes = [vp]
        L.orc_bwt_sa.restype = C.c_uint64
        L.orc_bwt_sa.argtypes = [vp, vp, C.c_uint64, C.c_uint64]
        L.orc_sa2pos.restype = C.c_uint64
        L.orc_sa2pos.argtypes = [vp, vp, C.c_uint64, C.c_uint64, C.c_int, ip]
        L.orc_suffix_array.argtypes = [vp, C.c_uint64, vp]
        L.orc_index_files.argtypes = [vp, C.c_uint64, C.c_char_p]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class Index:
    def __init__(self, bwt_path: str | None = None, file_words: np.ndarray | None = None):
        """A .bwt file, or its image in memory as uint32 words (kept alive here, not copied)."""
        err = C.c_int(0)
        if file_words is not None:
            self._words = np.ascontiguousarray(file_words, np.uint32)
            self.h = lib().orc_index_borrow(_ptr(self._words), len(self._words), C.byref(err))
        else:
            self.h = lib().orc_index_load(bwt_path.encode(), C.byref(err))
        if not self.h:
            raise IOError(f"cannot load {bwt_path or 'the .bwt image'} ({err.value})")
        prim, words = C.c_uint64(), C.c_uint64()
        L2 = (C.c_uint64 * 5)()
        lib().orc_index_meta(self.h, C.byref(prim), L2, C.byref(words))
        self.primary, self.L2, self.words = prim.value, list(L2), words.value

    def occ4(self, rows) -> np.ndarray:
        """Occ of the four bases at each row (the $ row not counted; ~0 = row -1): (n, 4) uint64."""
        k = np.ascontiguousarray(rows, np.uint64)
        out = np.zeros((max(1, len(k)), 4), np.uint64)
        lib().orc_occ4(self.h, _ptr(k), len(k), _ptr(out))
        return out[:len(k)]

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_index_free(self.h)
            self.h = None


def load_sa(prefix: str):
    """<prefix>.sa as bwt_restore_sa reads it (bwa's bwt.c:421-441): (samples with samples[0] = -1, interval)."""
    raw = np.fromfile(prefix + ".sa", dtype=np.uint64)
    intv, seq_len = int(raw[5]), int(raw[6])
    n_sa = (seq_len + intv) // intv
    samples = np.empty(n_sa, np.uint64)
    samples[0] = np.uint64(2**64 - 1)
    samples[1:] = raw[7:7 + n_sa - 1]
    return samples, intv


def bwt_sa(index: "Index", samples: np.ndarray, intv: int, rows) -> np.ndarray:
    """bwt_sa of each row (the oracle's restatement)."""
    L = lib()
    sp = np.ascontiguousarray(samples, np.uint64)
    return np.array([L.orc_bwt_sa(index.h, sp.ctypes.data, intv, int(k)) for k in rows], np.uint64)


def sa2pos(index: "Index", samples: np.ndarray, intv: int, rows, ref_len):
    """bwa_sa2pos of each (row, ref_len): (positions, strands)."""
    L = lib()
    sp = np.ascontiguousarray(samples, np.uint64)
    pos, strand = [], []
    st = C.c_int(0)
    for k, rl in zip(rows, ref_len):
        pos.append(L.orc_sa2pos(index.h, sp.ctypes.data, intv, int(k), int(rl), C.byref(st)))
        strand.append(st.value)
    return np.array(pos, np.uint64), np.array(strand, np.int8)


def load_reads(path: str) -> dict:
    """Reads of a FASTQ/FASTA file with the reference's rules: encoded queries, offsets, lengths, batch ids."""
    n, tot, err = C.c_int(), C.c_int64(), C.c_int()
    h = lib().orc_reads_load(path.encode(), C.byref(n), C.byref(tot), C.byref(err))
    if not h:
        raise IOError(f"cannot read {path} ({err.value})")
    q = np.zeros(max(1, tot.value), np.uint8)
    off = np.zeros(n.value + 1, np.int64)
    ln = np.zeros(max(1, n.value), np.int32)
    bt = np.zeros(max(1, n.value), np.int32)
    lib().orc_reads_get(h, _ptr(q), _ptr(off), _ptr(ln), _ptr(bt))
    lib().orc_reads_free(h)
    return dict(query=q[:tot.value], off=off, len=ln[:n.value], batch=bt[:n.value])


def encode_queries(ascii_seqs: np.ndarray, off: np.ndarray) -> np.ndarray:
    """query[j] = complement(nt4(read[len-1-j])), ambiguous -> 4 (host_io.c:178-183)"""
    nt4 = np.full(256, 4, np.uint8)
    for i, c in enumerate(b"ACGT"):
        nt4[c] = nt4[c + 32] = i
    codes = nt4[ascii_seqs]
    q = np.where(codes > 3, 4, 3 - codes).astype(np.uint8)
    out = np.empty_like(q)
    for r in range(len(off) - 1):
        s, e = int(off[r]), int(off[r + 1])
        out[s:e] = q[s:e][::-1]
    return out


def batches_for(n: int) -> np.ndarray:
    return (np.arange(n) // 0x40000).astype(np.int32)


class Result:
    def __init__(self, h, n):
        self.h, self.n = h, n
        L = lib()
        tot = L.orc_result_total(h)
        self.n_aln = np.zeros(max(1, n), np.int32)
        self.pops = np.zeros(max(1, n), np.uint64)
        self.trace = np.zeros(max(1, n), np.uint64)
        self.peak = np.zeros(max(1, n), np.int32)
        self.fetch128 = np.zeros(max(1, n), np.uint64)
        self.fetch64 = np.zeros(max(1, n), np.uint64)
        self.n_stacks = np.zeros(max(1, n), np.int32)
        self.max_diff = np.zeros(max(1, n), np.int32)
        self.rec_off = np.zeros(n + 1, np.int64)
        self.records = np.zeros(max(1, tot), REC_DTYPE)
        L.orc_result_dump(h, _ptr(self.n_aln), _ptr(self.pops), _ptr(self.trace), _ptr(self.peak),
                          _ptr(self.fetch128), _ptr(self.fetch64), _ptr(self.n_stacks), _ptr(self.max_diff),
                          _ptr(self.rec_off), _ptr(self.records))
        self.fetch80 = np.zeros(max(1, n), np.uint64)
        L.orc_result_fetch80(h, _ptr(self.fetch80))
        for a in ("n_aln", "pops", "trace", "peak", "fetch128", "fetch64", "fetch80", "n_stacks", "max_diff"):
            setattr(self, a, getattr(self, a)[:n])
        self.records = self.records[:tot]

    def write_sai(self, opt: bytes, path: str) -> int:
        return lib().orc_result_write_sai(self.h, opt, path.encode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_result_free(self.h)
            self.h = None


def aln(index: Index, opt: bytes, query, off, length, batch, n_threads: int = 0, batch_max_len=None) -> Result:
    n = len(length)
    q = np.ascontiguousarray(query, np.uint8)
    if q.size == 0:
        q = np.zeros(1, np.uint8)
    off = np.ascontiguousarray(off, np.int64)
    ln = np.ascontiguousarray(length, np.int32)
    bt = np.ascontiguousarray(batch, np.int32)
    nt = n_threads or max(1, os.cpu_count() or 1)
    if batch_max_len is None:
        h = lib().orc_aln(index.h, opt, _ptr(q), _ptr(off), _ptr(ln), _ptr(bt), n, nt)
    else:
        bm = np.ascontiguousarray(batch_max_len, np.int32)
        h = lib().orc_aln_bmax(index.h, opt, _ptr(q), _ptr(off), _ptr(ln), _ptr(bt), n, nt, _ptr(bm), len(bm))
    return Result(h, n)


def cal_maxdiff(l: int, err: float, thres: float) -> int:
    return lib().orc_cal_maxdiff(l, err, thres)


# ------------------------------------------------------------------------------------------------
# the reference itself

def run_galn_ref(prefix: str, fastq: str, args: list[str], out_sai: str, workers: int | None = None,
                 timeout: float = 3600.0, mode: str = "--cpu-only") -> dict:
    """Runs the reference's `galn aln --cpu-only` (or `--gpu-only`, its own GPU path) and returns its exit
    code and timing line."""
    cmd = [GALN_REF, "aln", mode] + list(args)
    if workers:
        cmd += ["--cpu-workers", str(workers)]
    cmd += ["-f", out_sai, prefix, fastq]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    info = dict(rc=p.returncode, stderr=p.stderr)
    for line in p.stderr.splitlines():
        if "search" in line and "reads" in line and "load" in line:
            # "[galn] N reads (...) in T s: load A s, search B s, write C s"
            try:
                info["search_s"] = float(line.split("search ")[1].split(" s")[0])
                info["n_reads"] = int(line.split("] ")[1].split(" reads")[0])
            except (IndexError, ValueError):
                pass
    return info


def ref_dump(bwt_path: str, fastq: str, opt: bytes, out_path: str, n_threads: int = 0) -> dict:
    """Per-read n_aln, records, pops and trace of the reference's aln_search_host."""
    L = C.CDLL(DUMP_REF)
    L.galnref_dump.restype = C.c_long
    L.galnref_dump.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_char_p]
    nt = n_threads or max(1, os.cpu_count() or 1)
    ret = L.galnref_dump(bwt_path.encode(), fastq.encode(), opt, nt, out_path.encode())
    if ret < 0:
        raise IOError(f"reference dump failed ({ret})")
    return parse_dump(out_path)


def parse_dump(path: str) -> dict:
    data = open(path, "rb").read()
    n = struct.unpack_from("<q", data, 0)[0]
    pos = 8
    hdr = np.dtype([("n", "<i4"), ("batch", "<i4"), ("len", "<i4"), ("peak", "<i4"), ("pops", "<u8"),
                    ("trace", "<u8"), ("n_stacks", "<i4"), ("max_diff", "<i4")])
    hs = np.zeros(n, hdr)
    recs = []
    rec_off = np.zeros(n + 1, np.int64)
    for r in range(n):
        h = np.frombuffer(data, hdr, 1, pos)[0]
        hs[r] = h
        pos += hdr.itemsize
        k = max(0, int(h["n"]))
        if k:
            recs.append(np.frombuffer(data, REC_DTYPE, k, pos))
            pos += 24 * k
        rec_off[r + 1] = rec_off[r] + k
    records = np.concatenate(recs) if recs else np.zeros(0, REC_DTYPE)
    return dict(n_aln=hs["n"], batch=hs["batch"], len=hs["len"], peak=hs["peak"], pops=hs["pops"],
                trace=hs["trace"], n_stacks=hs["n_stacks"], max_diff=hs["max_diff"], rec_off=rec_off,
                records=records)


def read_sai(path: str) -> dict:
    """Parses a .sai stream: option block and per-read records."""
    data = open(path, "rb").read()
    assert data[:4] == b"SAI\x01", "not a .sai file"
    opt = data[4:68]
    pos = 68
    ns, recs = [], []
    while pos < len(data):
        k = struct.unpack_from("<i", data, pos)[0]
        pos += 4
        ns.append(k)
        if k > 0:
            recs.append(np.frombuffer(data, REC_DTYPE, k, pos))
            pos += 24 * k
    return dict(opt=opt, n_aln=np.array(ns, np.int32),
                records=np.concatenate(recs) if recs else np.zeros(0, REC_DTYPE))


# ------------------------------------------------------------------------------------------------
# index files (bwa index 0.7.19 .bwt / .sa; src/index/idxcommon.c:72-153)

def suffix_array(T: np.ndarray) -> np.ndarray:
    """SA of T$ (codes 0..3) over its n+1 rows; row 0 is the $ suffix (position n). Comparison sort."""
    t = np.ascontiguousarray(T, dtype=np.uint8)
    sa = np.zeros(len(t) + 1, dtype=np.uint64)
    lib().orc_suffix_array(_ptr(t), len(t), _ptr(sa))
    return sa


def index_files(F: np.ndarray, prefix: str) -> None:
    """<prefix>.bwt and <prefix>.sa for the forward sequence F (codes 0..3), as bwa index writes them."""
    f = np.ascontiguousarray(F, dtype=np.uint8)
    if lib().orc_index_files(_ptr(f), len(f), prefix.encode()):
        raise RuntimeError("orc_index_files failed")


def forward_from_pac(pac_path: str) -> np.ndarray:
    """The forward sequence (codes 0..3) held in a .pac file: 4 bases a byte, the first in the top bits; the
    last byte holds l_pac % 4 (after a 0 byte when that is 0)."""
    b = np.fromfile(pac_path, dtype=np.uint8)
    rem = int(b[-1])
    nbytes = len(b) - (2 if rem == 0 else 1)
    codes = np.stack([(b[:nbytes] >> s) & 3 for s in (6, 4, 2, 0)], axis=1).reshape(-1)
    l_pac = nbytes * 4 if rem == 0 else (nbytes - 1) * 4 + rem
    return codes[:l_pac].astype(np.uint8)
