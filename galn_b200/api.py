"""ctypes binding of include/galn_aln.h and the Python mirror of the `galn aln` interface."""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

GALN_ENGINE_PLAIN = 0
GALN_ENGINE_PERSISTENT = 1
REC_DTYPE = np.dtype([("packed", "<u8"), ("k", "<u8"), ("l", "<u8")])


class GalnError(RuntimeError):
    pass


class Options(C.Structure):
    """gap_opt_t: the 64-byte option block written into the .sai header."""
    _fields_ = [("s_mm", C.c_int32), ("s_gapo", C.c_int32), ("s_gape", C.c_int32), ("mode", C.c_int32),
                ("indel_end_skip", C.c_int32), ("max_del_occ", C.c_int32), ("max_entries", C.c_int32),
                ("fnr", C.c_float), ("max_diff", C.c_int32), ("max_gapo", C.c_int32), ("max_gape", C.c_int32),
                ("max_seed_diff", C.c_int32), ("seed_len", C.c_int32), ("n_threads", C.c_int32),
                ("max_top2", C.c_int32), ("trim_qual", C.c_int32)]


class _Reads(C.Structure):
    _fields_ = [("n_reads", C.c_int32), ("seq", C.c_void_p), ("offset", C.c_void_p), ("batch", C.c_void_p),
                ("batch_max_len", C.c_void_p), ("n_batches", C.c_int32)]


class _ReadSet(C.Structure):
    _fields_ = [("reads", _Reads), ("names", C.POINTER(C.c_char_p)), ("_priv", C.c_void_p)]


class _Results(C.Structure):
    _fields_ = [("n_reads", C.c_int32), ("n_aln", C.POINTER(C.c_int32)), ("rec_offset", C.POINTER(C.c_int64)),
                ("rec", C.c_void_p), ("n_pops", C.POINTER(C.c_uint64)), ("trace", C.POINTER(C.c_uint64)),
                ("_priv", C.c_void_p)]


class BuildStats(C.Structure):
    _fields_ = [("n", C.c_uint64), ("primary", C.c_uint64), ("rounds", C.c_int), ("sort_passes", C.c_int),
                ("sorted_items", C.c_uint64), ("scatter_items", C.c_uint64), ("ms_device", C.c_double),
                ("ms_copies", C.c_double), ("ms_scatter", C.c_double), ("ms_files", C.c_double)]


def lib_path() -> str:
    return os.path.join(HERE, "libgalnb200.so")


_lib = None


def lib():
    """The loaded library; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    p = lib_path()
    if not os.path.exists(p):
        raise GalnError(f"{p} is missing: build it with `python -m galn_b200.build` (no CPU fallback exists)")
    L = C.CDLL(p)
    vp = C.c_void_p
    L.galn_opts_default.argtypes = [C.POINTER(Options)]
    L.galn_opts_parse.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(Options), C.POINTER(C.c_char_p), C.c_int,
                                  C.POINTER(C.c_int), C.POINTER(C.c_char_p), C.c_char_p, C.c_size_t]
    L.galn_cal_maxdiff.argtypes = [C.c_int, C.c_double, C.c_double]
    L.galn_index_open.restype = vp
    L.galn_index_open.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int)]
    L.galn_index_open_mem.restype = vp
    L.galn_index_open_mem.argtypes = [vp, C.c_size_t, C.c_int, C.POINTER(C.c_int)]
    L.galn_index_close.argtypes = [vp]
    L.galn_index_info.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.galn_fastq_read.argtypes = [C.c_char_p, C.POINTER(_ReadSet)]
    L.galn_read_set_free.argtypes = [C.POINTER(_ReadSet)]
    L.galn_fastq_open.restype = vp
    L.galn_fastq_open.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
    L.galn_fastq_next.argtypes = [vp, C.POINTER(_ReadSet)]
    L.galn_fastq_close.argtypes = [vp]
    L.galn_index_load_sa.argtypes = [vp, C.c_char_p]
    L.galn_bwt_sa.argtypes = [vp, vp, C.c_int64, vp]
    L.galn_sa2pos.argtypes = [vp, vp, vp, C.c_int64, vp, vp]
    L.galn_results_free.argtypes = [C.POINTER(_Results)]
    L.galn_aln_run_batch.argtypes = [vp, C.POINTER(Options), C.POINTER(_Reads), C.c_int, C.POINTER(_Results)]
    L.galn_sai_write.argtypes = [C.c_char_p, C.POINTER(Options), C.POINTER(_Results)]
    L.galn_last_run_stats.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.galn_last_run_profile.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), vp, vp, vp, vp, C.c_int32]
    L.galn_index_set_tuning.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    L.galn_index_set_trace.argtypes = [vp, C.c_int]
    L.galn_index_set_warp_tier.argtypes = [vp, C.c_int, C.c_int]
    L.galn_last_warp_counters.argtypes = [vp, vp, C.c_int]
    L.galn_server_start.restype = vp
    L.galn_server_start.argtypes = [vp, C.c_size_t, C.POINTER(C.c_int)]
    L.galn_server_stop.argtypes = [vp]
    L.galn_server_configure.argtypes = [vp, C.c_int, C.c_int]
    L.galn_aln_submit.restype = C.c_int64
    L.galn_aln_submit.argtypes = [vp, C.POINTER(Options), C.POINTER(_Reads)]
    L.galn_aln_wait.argtypes = [vp, C.c_int64, C.c_int, C.POINTER(_Results)]
    L.galn_server_stats.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    L.galn_autotune.argtypes = [vp, C.POINTER(Options), C.POINTER(_Reads), C.c_int, C.POINTER(C.c_int),
                                C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.galn_autotune_clear.argtypes = [vp]
    L.galn_autotune_choice.argtypes = [vp, C.POINTER(Options), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.galn_last_graph_launches.argtypes = [vp, C.POINTER(C.c_int64)]
    L.galn_index_build_text.argtypes = [vp, C.c_uint64, C.c_char_p, C.c_int, C.POINTER(BuildStats)]
    L.galn_index_build_text_ex.argtypes = [vp, C.c_uint64, C.c_char_p, C.c_int, C.c_int64, C.POINTER(BuildStats)]
    L.galn_index_build_fasta.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(BuildStats)]
    L.galn_fasta_to_pac.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_uint64)]
    L.galn_gather_peak.argtypes = [C.c_int, C.c_uint64, C.c_int, C.POINTER(C.c_double)]
    L.galn_index_set_warp_wait.argtypes = [vp, C.c_int64]
    L.galn_index_set_fused.argtypes = [vp, C.c_int]
    L.galn_index_set_warp_order.argtypes = [vp, C.c_int]
    L.galn_last_run_fused.argtypes = [vp, C.POINTER(C.c_int)]
    L.galn_index_occ.argtypes = [vp, C.c_int, vp, C.c_int64, vp, vp]
    L.galn_stack_need.argtypes = [vp, C.POINTER(Options), C.POINTER(_Reads), C.POINTER(C.c_uint64)]
    L.galn_server_memory.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_int64)]
    L.galn_server_admissions.argtypes = [vp, vp, C.c_int]
    L.galn_last_warp_queue.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int)]
    L.galn_gather_peak_ex.argtypes = [C.c_int, C.c_uint64, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.galn_version.restype = C.c_char_p
    _lib = L
    return L


def parse_options(args: list[str]) -> Options:
    """The option block of `galn aln <args>` (positional arguments are not allowed here)."""
    o = Options()
    argv = (C.c_char_p * max(1, len(args)))(*[a.encode() for a in args])
    pos = (C.c_char_p * 4)()
    npos = C.c_int(0)
    outp = C.c_char_p()
    err = C.create_string_buffer(256)
    rc = lib().galn_opts_parse(len(args), argv, C.byref(o), pos, 4, C.byref(npos), C.byref(outp), err, 256)
    if rc != 0:
        raise GalnError(err.value.decode())
    if npos.value:
        raise GalnError("unexpected positional argument")
    return o


def cal_maxdiff(length: int, err: float, thres: float) -> int:
    return lib().galn_cal_maxdiff(length, err, thres)


class Index:
    """<prefix>.bwt resident on one GPU in the device occurrence layout."""

    def __init__(self, prefix: str | None = None, device: int = 0, bwt_bytes: bytes | np.ndarray | None = None):
        """<prefix>.bwt, or a .bwt file's image in memory (bytes, or a numpy array used without a copy)."""
        err = C.c_int(0)
        if isinstance(bwt_bytes, np.ndarray):
            a = np.ascontiguousarray(bwt_bytes)
            self.h = lib().galn_index_open_mem(a.ctypes.data, a.nbytes, device, C.byref(err))
        elif bwt_bytes is not None:
            buf = C.create_string_buffer(bwt_bytes, len(bwt_bytes))
            self.h = lib().galn_index_open_mem(buf, len(bwt_bytes), device, C.byref(err))
        else:
            self.h = lib().galn_index_open(prefix.encode(), device, C.byref(err))
        if not self.h:
            raise GalnError(f"cannot open the index ({err.value})")
        n, p, b = C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib().galn_index_info(self.h, C.byref(n), C.byref(p), C.byref(b))
        self.seq_len, self.primary, self.device_bytes = n.value, p.value, b.value

    def close(self):
        if getattr(self, "h", None):
            lib().galn_index_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_tuning(self, t0_cap=1024, t0_aln=32, t0_block=128, t1_cap=65536, t1_aln=1024, keep_stats=False):
        rc = lib().galn_index_set_tuning(self.h, t0_cap, t0_aln, t0_block, t1_cap, t1_aln, int(keep_stats))
        if rc:
            raise GalnError(f"bad tuning ({rc})")

    def set_warp_tier(self, on: bool, arena_chunks: int = 1 << 13):
        if lib().galn_index_set_warp_tier(self.h, int(on), arena_chunks):
            raise GalnError("bad warp tier setting")

    def set_warp_order(self, order: int):
        """Order of the heavy reads handed to the warp tier (galn_index_set_warp_order)."""
        if lib().galn_index_set_warp_order(self.h, int(order)):
            raise GalnError("bad warp order")

    def set_fused(self, on: bool):
        """The persistent engine's first and warp tiers as one launch (galn_index_set_fused) for option sets the
        autotuner has not tuned; off by default (two launches)."""
        if lib().galn_index_set_fused(self.h, int(on)):
            raise GalnError("bad fused setting")

    def set_warp_wait(self, wait_ns: int):
        """How long a big-arena warp waits for queued reads (galn_index_set_warp_wait; default 2 s)."""
        if lib().galn_index_set_warp_wait(self.h, int(wait_ns)):
            raise GalnError("bad warp wait")

    def last_warp_queue(self) -> dict:
        """Reads the last run's warp tier queued for its big-arena warps, and whether a wait ran out."""
        q, g = C.c_int64(), C.c_int()
        lib().galn_last_warp_queue(self.h, C.byref(q), C.byref(g))
        return dict(queued=q.value, gave_up=bool(g.value))

    def load_sa(self, prefix: str):
        """Put <prefix>.sa (the suffix-array samples of this index) on the device for positions."""
        rc = lib().galn_index_load_sa(self.h, prefix.encode())
        if rc:
            raise GalnError(f"cannot load {prefix}.sa ({rc})")

    def bwt_sa(self, rows) -> np.ndarray:
        """bwt_sa of each suffix-array row (the forward-reverse coordinate; row 0 gives 2**64 - 1)."""
        k = np.ascontiguousarray(rows, np.uint64)
        out = np.zeros(max(1, len(k)), np.uint64)
        rc = lib().galn_bwt_sa(self.h, k.ctypes.data, len(k), out.ctypes.data)
        if rc:
            raise GalnError(f"galn_bwt_sa failed ({rc})")
        return out[:len(k)]

    def sa2pos(self, rows, ref_len):
        """bwa_sa2pos of each (row, reference length of the hit): (positions, strands)."""
        k = np.ascontiguousarray(rows, np.uint64)
        rl = np.ascontiguousarray(ref_len, np.int32)
        pos = np.zeros(max(1, len(k)), np.uint64)
        strand = np.zeros(max(1, len(k)), np.int8)
        rc = lib().galn_sa2pos(self.h, k.ctypes.data, rl.ctypes.data, len(k), pos.ctypes.data, strand.ctypes.data)
        if rc:
            raise GalnError(f"galn_sa2pos failed ({rc})")
        return pos[:len(k)], strand[:len(k)]

    def occ(self, rows, layout: int = 64) -> np.ndarray:
        """Occ of the four bases at each BWT row (galn_index_occ): an (n, 4) uint64 array."""
        k = np.ascontiguousarray(rows, np.uint64)
        out = np.zeros((max(1, len(k)), 4), np.uint64)
        rc = lib().galn_index_occ(self.h, layout, k.ctypes.data, len(k), out.ctypes.data, None)
        if rc:
            raise GalnError(f"galn_index_occ failed ({rc})")
        return out[:len(k)]

    def info(self) -> dict:
        n, p, b = C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib().galn_index_info(self.h, C.byref(n), C.byref(p), C.byref(b))
        return dict(seq_len=n.value, primary=p.value, device_bytes=b.value)

    def set_l2_persist(self, on: bool):
        """Keep the occurrence blocks in a persisting L2 window (on by default)."""
        if lib().galn_index_set_l2_persist(self.h, int(on)):
            raise GalnError("bad L2 setting")

    def warp_counters(self) -> dict:
        v = np.zeros(15, np.uint64)
        lib().galn_last_warp_counters(self.h, v.ctypes.data, 15)
        names = ["reads", "waves", "lanes", "consumed", "pops", "continued", "hits", "cyc_chain", "cyc_replay",
                 "cyc_commit", "cyc_load", "chain_pops", "cyc_read", "steps", "cyc_read_max"]
        return {k: int(x) for k, x in zip(names, v)}

    def autotune(self, args, reads: "Reads", max_sample: int = 131072) -> dict:
        """Pick the occurrence layout, first-tier stack depth and block size for these options on a sample of
        `reads`."""
        opts = args if isinstance(args, Options) else parse_options(list(args))
        cr, keep = reads.c_struct()
        cap, blk, occ, ms = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        rc = lib().galn_autotune(self.h, C.byref(opts), C.byref(cr), max_sample, C.byref(cap), C.byref(blk),
                                 C.byref(occ), C.byref(ms))
        if rc:
            raise GalnError(f"autotune failed ({rc})")
        arena, big, div = C.c_int(), C.c_int(), C.c_int()
        lib().galn_autotune_choice(self.h, C.byref(opts), None, None, None, C.byref(arena), C.byref(big), C.byref(div))
        return dict(t0_cap=cap.value, block=blk.value, occ=occ.value, warp_arena=arena.value, warp_big=big.value,
                    fused_div=div.value, ms=ms.value)

    def set_occ_layout(self, stride: int):
        """Occurrence layout (64 or 80 symbols per 32-byte block) when the autotuner has no choice."""
        if lib().galn_index_set_occ_layout(self.h, stride):
            raise GalnError("bad occ layout")

    def set_trace(self, on: bool):
        lib().galn_index_set_trace(self.h, int(on))

    def last_profile(self, n: int = 0) -> dict:
        """Device span and per-tier kernel ms of the last run; with n > 0 (and keep_stats tuning) also the
        per-read 32-byte block fetches and finishing tier."""
        dev = C.c_double()
        tiers = (C.c_double * 8)()
        treads = np.zeros(8, np.int64)
        tthreads = np.zeros(8, np.int64)
        fetch = np.zeros(max(n, 1), np.uint32)
        tier = np.zeros(max(n, 1), np.int8)
        rc = lib().galn_last_run_profile(self.h, C.byref(dev), tiers, treads.ctypes.data, tthreads.ctypes.data,
                                         fetch.ctypes.data if n else None, tier.ctypes.data if n else None, n)
        if rc:
            raise GalnError(f"no profile ({rc})")
        fused = C.c_int(0)
        lib().galn_last_run_fused(self.h, C.byref(fused))
        out = dict(ms_device=dev.value, ms_tier=list(tiers), tier_reads=treads.tolist(),
                   tier_threads=tthreads.tolist(), fused=bool(fused.value))
        if n:
            out["fetch"] = fetch[:n]
            out["tier"] = tier[:n]
        return out

    def last_phases(self) -> dict:
        """Host-side timeline of the last run, in ms from the call's start."""
        v = (C.c_double * 8)()
        lib().galn_last_run_phases(self.h, v, 8)
        return dict(launch=v[0], device_done=v[1], results=v[2], total=v[3], device=v[4], first_tier_done=v[5],
                    warp_launch=v[6], first_tier_launch=v[7])

    def last_stats(self) -> dict:
        t, k, tiers, la = C.c_double(), C.c_double(), C.c_int(), C.c_int64()
        ovf = (C.c_int64 * 8)()
        lib().galn_last_run_stats(self.h, C.byref(t), C.byref(k), C.byref(tiers), C.byref(la), ovf)
        g = C.c_int64()
        lib().galn_last_graph_launches(self.h, C.byref(g))
        return dict(ms_total=t.value, ms_kernels=k.value, tiers=tiers.value, launches=la.value, overflow=list(ovf),
                    graph_launches=g.value)


@dataclass
class Reads:
    """ASCII bases concatenated (uint8), n+1 int64 offsets, optional int32 batch ids."""
    seq: np.ndarray
    offset: np.ndarray
    batch: np.ndarray | None = None
    batch_max_len: np.ndarray | None = None
    names: list[str] | None = None

    def __len__(self):
        return len(self.offset) - 1

    @staticmethod
    def from_strings(seqs: list[str | bytes]) -> "Reads":
        bs = [s.encode() if isinstance(s, str) else s for s in seqs]
        off = np.zeros(len(bs) + 1, np.int64)
        off[1:] = np.cumsum([len(b) for b in bs])
        return Reads(np.frombuffer(b"".join(bs) or b"\0", np.uint8)[:off[-1]].copy(), off)

    def c_struct(self) -> tuple[_Reads, list]:
        keep = []
        seq = np.ascontiguousarray(self.seq, np.uint8)
        if seq.size == 0:
            seq = np.zeros(1, np.uint8)
        off = np.ascontiguousarray(self.offset, np.int64)
        keep += [seq, off]
        r = _Reads()
        r.n_reads = len(off) - 1
        r.seq = seq.ctypes.data
        r.offset = off.ctypes.data
        if self.batch is not None:
            b = np.ascontiguousarray(self.batch, np.int32)
            keep.append(b)
            r.batch = b.ctypes.data
        if self.batch_max_len is not None:
            m = np.ascontiguousarray(self.batch_max_len, np.int32)
            keep.append(m)
            r.batch_max_len = m.ctypes.data
            r.n_batches = len(m)
        return r, keep


def _reads_from_set(rs: _ReadSet) -> Reads:
    n = rs.reads.n_reads
    off = np.ctypeslib.as_array(C.cast(rs.reads.offset, C.POINTER(C.c_int64)), (n + 1,)).copy()
    total = int(off[-1])
    seq = (np.ctypeslib.as_array(C.cast(rs.reads.seq, C.POINTER(C.c_uint8)), (total,)).copy()
           if total else np.zeros(0, np.uint8))
    batch = (np.ctypeslib.as_array(C.cast(rs.reads.batch, C.POINTER(C.c_int32)), (n,)).copy()
             if n else np.zeros(0, np.int32))
    names = [rs.names[i].decode() for i in range(n)]
    lib().galn_read_set_free(C.byref(rs))
    return Reads(seq, off, batch, None, names)


def read_fastq(path: str) -> Reads:
    """A FASTQ/FASTA file read by the library with the reference's rules (batch ids included)."""
    rs = _ReadSet()
    rc = lib().galn_fastq_read(path.encode(), C.byref(rs))
    if rc != 0:
        raise GalnError(f"cannot read {path} ({rc})")
    return _reads_from_set(rs)


def read_fastq_batches(path: str):
    """The same reads one bwa batch at a time (a generator of Reads; batch ids as in the whole file)."""
    err = C.c_int(0)
    st = lib().galn_fastq_open(path.encode(), C.byref(err))
    if not st:
        raise GalnError(f"cannot read {path} ({err.value})")
    try:
        while True:
            rs = _ReadSet()
            rc = lib().galn_fastq_next(st, C.byref(rs))
            if rc != 0:
                raise GalnError(f"cannot read {path} ({rc})")
            if rs.reads.n_reads == 0:
                lib().galn_read_set_free(C.byref(rs))
                return
            yield _reads_from_set(rs)
    finally:
        lib().galn_fastq_close(st)


class _ResultsOwner:
    """Owns a galn_results of the library; freed when the last array viewing it is gone."""

    def __init__(self, r: _Results):
        self.r = r

    def __del__(self):
        try:
            lib().galn_results_free(C.byref(self.r))
        except Exception:   # noqa: BLE001 -- interpreter shutdown
            pass


def _view(owner: _ResultsOwner, addr: int, ctype, n: int, dtype) -> np.ndarray:
    """A numpy array over n items of the owner's memory at addr; it keeps the owner alive."""
    buf = (ctype * n).from_address(addr)
    buf._owner = owner
    return np.frombuffer(buf, dtype)


class Results:
    """Per-read results of one search. The arrays are views of the library's result memory (no copy); it is
    freed when the Results and every array taken from it are gone."""

    def __init__(self, r: _Results, opts: Options):
        n = r.n_reads
        self.opts = opts
        if n == 0:
            lib().galn_results_free(C.byref(r))
            self.n_aln = np.zeros(0, np.int32)
            self.rec_offset = np.zeros(1, np.int64)
            self.records = np.zeros(0, REC_DTYPE)
            self.pops = np.zeros(0, np.uint64)
            self.trace = np.zeros(0, np.uint64)
            return
        owner = _ResultsOwner(r)
        self.n_aln = _view(owner, C.cast(r.n_aln, C.c_void_p).value, C.c_int32, n, np.int32)
        self.rec_offset = _view(owner, C.cast(r.rec_offset, C.c_void_p).value, C.c_int64, n + 1, np.int64)
        tot = int(self.rec_offset[-1])
        self.records = _view(owner, r.rec, C.c_char, 24 * tot, REC_DTYPE) if tot else np.zeros(0, REC_DTYPE)
        self.pops = _view(owner, C.cast(r.n_pops, C.c_void_p).value, C.c_uint64, n, np.uint64)
        self.trace = _view(owner, C.cast(r.trace, C.c_void_p).value, C.c_uint64, n, np.uint64)

    def __len__(self):
        return len(self.n_aln)

    def sai_bytes(self) -> bytes:
        """The .sai stream: header, then per read int32 n_aln (0 for an error code) and its records."""
        n = len(self.n_aln)
        na = np.maximum(self.n_aln, 0).astype(np.int64)
        tot = int(na.sum())
        hdr = b"SAI\x01" + bytes(self.opts)
        out = np.empty(len(hdr) + 4 * n + 24 * tot, np.uint8)
        out[:len(hdr)] = np.frombuffer(hdr, np.uint8)
        first = np.zeros(n + 1, np.int64)            # each read's first record in the output order
        first[1:] = np.cumsum(na)
        at = len(hdr) + 4 * np.arange(n, dtype=np.int64) + 24 * first[:-1]
        out[at[:, None] + np.arange(4)] = na.astype(np.int32).view(np.uint8).reshape(n, 4)
        if tot:
            owner = np.repeat(np.arange(n), na)
            src = np.repeat(self.rec_offset[:-1], na) + (np.arange(tot) - np.repeat(first[:-1], na))
            dst = len(hdr) + 4 * (owner + 1) + 24 * np.arange(tot, dtype=np.int64)
            out[dst[:, None] + np.arange(24)] = self.records[src].view(np.uint8).reshape(tot, 24)
        return out.tobytes()

    def write_sai(self, path: str) -> int:
        with open(path, "wb") as f:
            f.write(self.sai_bytes())
        return 4 if (self.n_aln < 0).any() else 0


def aln(index: Index, args: list[str] | Options, reads: Reads | str,
        engine: int = GALN_ENGINE_PERSISTENT) -> Results:
    """`galn aln <args>` on the reads (a Reads object or a FASTQ path) against a resident index."""
    opts = args if isinstance(args, Options) else parse_options(list(args))
    if isinstance(reads, str):
        reads = read_fastq(reads)
    cr, keep = reads.c_struct()
    res = _Results()
    rc = lib().galn_aln_run_batch(index.h, C.byref(opts), C.byref(cr), engine, C.byref(res))
    if rc != 0:
        raise GalnError(f"galn_aln_run_batch failed ({rc})")
    out = Results(res, opts)   # takes ownership of the library's result memory
    del keep
    return out


def write_sai(path: str, res: Results) -> int:
    return res.write_sai(path)


def gather_peak(device: int, nbytes: int, in_flight: int = 8, repeats: int = 5) -> float | None:
    """Random 32-byte sector read rate (GB/s) over a buffer of nbytes (galn_gather_peak_ex), or None."""
    g = C.c_double(0)
    rc = lib().galn_gather_peak_ex(device, nbytes, in_flight, repeats, C.byref(g))
    return g.value if rc == 0 else None


def _stats_dict(st: BuildStats) -> dict:
    return {f: getattr(st, f) for f, _ in BuildStats._fields_}


def index_fasta(fasta: str, prefix: str, device: int = 0) -> dict:
    """`galn index -p prefix fasta` on a CUDA device: the five bwa index files (galn_index_build_fasta).
    Returns the builder's statistics."""
    st = BuildStats()
    rc = lib().galn_index_build_fasta(fasta.encode(), prefix.encode(), device, C.byref(st))
    if rc:
        raise GalnError(f"galn_index_build_fasta failed ({rc})")
    return _stats_dict(st)


def fasta_to_pac(fasta: str, prefix: str) -> int:
    """The host step of `galn index`: <prefix>.pac/.ann/.amb from a FASTA file. Returns the reference length."""
    n = C.c_uint64()
    rc = lib().galn_fasta_to_pac(fasta.encode(), prefix.encode(), C.byref(n))
    if rc:
        raise GalnError(f"galn_fasta_to_pac failed ({rc})")
    return n.value


def index_text(fwd: np.ndarray, prefix: str, device: int = 0, sort_chunk: int = 0) -> dict:
    """<prefix>.bwt and <prefix>.sa for the forward sequence fwd (codes 0..3; the text is fwd . revcomp(fwd)),
    built on a CUDA device (galn_index_build_text_ex; sort_chunk > 0 takes the 64-bit path with at most that
    many suffixes sorted at once)."""
    f = np.ascontiguousarray(fwd, dtype=np.uint8)
    st = BuildStats()
    rc = lib().galn_index_build_text_ex(f.ctypes.data, len(f), prefix.encode(), device, sort_chunk, C.byref(st))
    if rc:
        raise GalnError(f"galn_index_build_text failed ({rc})")
    return _stats_dict(st)


class Server:
    """Continuous-batching request loop on a resident index (galn_server_*)."""

    def __init__(self, index: Index, stack_bytes: int = 0, step_reads: int | None = None, max_active: int = 64,
                 fill_reads: int = 0):
        err = C.c_int(0)
        self.index = index
        self.h = lib().galn_server_start(index.h, stack_bytes, C.byref(err))
        if not self.h:
            raise GalnError(f"cannot start the server ({err.value})")
        if step_reads is not None:
            lib().galn_server_configure(self.h, step_reads, max_active)
        if fill_reads:
            lib().galn_server_set_step_fill(self.h, fill_reads)
        self._keep = {}

    def submit(self, args: list[str] | Options, reads: Reads) -> int:
        opts = args if isinstance(args, Options) else parse_options(list(args))
        cr, keep = reads.c_struct()
        rid = lib().galn_aln_submit(self.h, C.byref(opts), C.byref(cr))
        if rid <= 0:
            raise GalnError(f"submit failed ({rid})")
        self._keep[rid] = opts
        return rid

    def wait(self, rid: int, timeout_ms: int = -1) -> Results:
        res = _Results()
        rc = lib().galn_aln_wait(self.h, rid, timeout_ms, C.byref(res))
        if rc != 0:
            raise GalnError(f"request {rid} failed ({rc})")
        out = Results(res, self._keep.pop(rid))   # takes ownership
        return out

    def stats(self) -> dict:
        p50, p99, busy = C.c_double(), C.c_double(), C.c_double()
        nr, nreads, steps = C.c_int64(), C.c_int64(), C.c_int64()
        lib().galn_server_stats(self.h, C.byref(p50), C.byref(p99), C.byref(nr), C.byref(nreads), C.byref(busy),
                                C.byref(steps))
        return dict(p50_ms=p50.value, p99_ms=p99.value, requests=nr.value, reads=nreads.value, busy_ms=busy.value,
                    steps=steps.value)

    def stack_need(self, args: list[str] | Options, reads: Reads) -> int:
        """Device memory the server reserves for this request's search stacks (galn_stack_need)."""
        opts = args if isinstance(args, Options) else parse_options(list(args))
        cr, keep = reads.c_struct()
        v = C.c_uint64()
        if lib().galn_stack_need(self.h, C.byref(opts), C.byref(cr), C.byref(v)):
            raise GalnError("galn_stack_need failed")
        return v.value

    def memory(self) -> dict:
        b, u, p, h = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_int64()
        lib().galn_server_memory(self.h, C.byref(b), C.byref(u), C.byref(p), C.byref(h))
        return dict(budget=b.value, in_use=u.value, peak=p.value, held_back=h.value)

    def admissions(self, n: int = 1 << 16) -> list[int]:
        """Request ids in the order they were admitted."""
        ids = np.zeros(max(1, n), np.int64)
        k = lib().galn_server_admissions(self.h, ids.ctypes.data, n)
        return ids[:max(0, k)].tolist()

    def close(self):
        if getattr(self, "h", None):
            lib().galn_server_stop(self.h)
            self.h = None

    def __del__(self):
        self.close()
