"""Builds galn-b200's native code in-tree for sm_100a:

    galn_b200/libgalnb200.so   the library behind include/galn_aln.h (CUDA kernels + C++ host)
    galn_b200/bin/galn         the `galn aln` command line

Objects go to galn_b200/_build/; each output has a stamp of the command and the contents of its inputs, and a
step runs again when the stamp differs (a changed source, header or flag), not when file times say so.
Host C++ is compiled with -ffp-contract=off so that bwa_cal_maxdiff rounds as the reference does.
"""
from __future__ import annotations

import glob
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgalnb200.so")
CLI = os.path.join(HERE, "bin", "galn")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
                  "-I" + os.path.join(ROOT, "include")]
CXXFLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-Wall", "-I" + os.path.join(CUDA, "include"),
            "-I" + os.path.join(ROOT, "include")]

CU_SOURCES = ["galn_kernels.cu", "galn_noalloc.cu", "galn_build_index.cu"]
CPP_SOURCES = ["galn_host.cpp", "galn_engine.cpp", "galn_serve.cpp", "galn_tune.cpp", "galn_index_files.cpp"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(ROOT, "include", "galn_aln.h")]


def _digest(cmd, deps):
    """SHA-1 of a build step: its command line and the bytes of every input, with the repository's own path
    left out, so that a copy of the tree elsewhere (its built files included) needs no rebuild."""
    h = hashlib.sha1("\0".join(cmd).replace(ROOT, "@").encode())
    for d in deps:
        h.update(os.path.relpath(d, ROOT).encode())
        if os.path.exists(d):
            with open(d, "rb") as f:
                h.update(f.read())
    return h.hexdigest()


def _step(target, cmd, deps, verbose):
    """Runs cmd unless target exists with a stamp (target + '.stamp') of the same command and inputs. The
    stamp is taken from the inputs as they were before the step ran, so an input edited while it ran makes
    the next build run it again (file times alone would call the result newer than the edit)."""
    stamp = target + ".stamp"
    want = _digest(cmd, deps)
    if os.path.exists(target) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == want:
                return
    if os.path.exists(stamp):
        os.remove(stamp)
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    with open(stamp, "w") as f:
        f.write(want + "\n")


def build(verbose: bool = False, extra_nvflags: list[str] | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = sorted(_headers())
    objs = []
    for s in CU_SOURCES:
        src, obj = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        _step(obj, [NVCC] + NVFLAGS + (extra_nvflags or []) + ["-c", src, "-o", obj], [src] + hdrs, verbose)
        objs.append(obj)
    for s in CPP_SOURCES:
        src, obj = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        _step(obj, ["g++"] + CXXFLAGS + ["-c", src, "-o", obj], [src] + hdrs, verbose)
        objs.append(obj)
    _step(LIB, [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lz", "-lpthread"], objs, verbose)
    main_src, main_obj = os.path.join(CSRC, "galn_main.cpp"), os.path.join(BUILD, "galn_main.cpp.o")
    _step(main_obj, ["g++"] + CXXFLAGS + ["-c", main_src, "-o", main_obj], [main_src] + hdrs, verbose)
    _step(CLI, ["g++", "-o", CLI, main_obj, "-L" + HERE, "-lgalnb200", "-Wl,-rpath,$ORIGIN/..",
                "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-lpthread"], [main_obj, LIB], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
