"""galn-b200: the `bwa aln` FM-index backtracking search on NVIDIA B200 (sm_100a).

The search runs in CUDA kernels behind the C ABI of include/galn_aln.h (libgalnb200.so, built in-tree by
galn_b200.build). This module binds that ABI with ctypes and mirrors the reference's `galn aln` surface:

    ix = galn_b200.Index("ref")                     # <prefix>.bwt onto the GPU
    res = galn_b200.aln(ix, ["-l", "1024", "-n", "0.01", "-o", "2"], reads)
    res.write_sai("out.sai")
    galn_b200.index_fasta("ref.fa", "ref")          # `galn index`: the bwa index files, built on the GPU

There is no CPU fallback: if the library is missing or no sm_100 device is present, the calls raise.
"""
from __future__ import annotations

from .api import (GALN_ENGINE_PERSISTENT, GALN_ENGINE_PLAIN, GalnError, Index, Options, Reads, Results,  # noqa: F401
                  Server, aln, cal_maxdiff, fasta_to_pac, gather_peak, index_fasta, index_text, lib, lib_path, parse_options,
                  read_fastq,
                  read_fastq_batches, write_sai)
