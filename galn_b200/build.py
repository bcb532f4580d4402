"""Builds galn-b200's native code in-tree for sm_100a:

    galn_b200/libgalnb200.so   the library behind include/galn_aln.h (CUDA kernels + C++ host)
    galn_b200/bin/galn         the `galn aln` command line

Objects go to galn_b200/_build/; a source is recompiled when it or any header is newer than its object.
Host C++ is compiled with -ffp-contract=off so that bwa_cal_maxdiff rounds as the reference does.
"""
from __future__ import annotations

import glob
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


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, extra_nvflags: list[str] | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = _headers()
    objs = []
    for s in CU_SOURCES:
        src, obj = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        if _stale(obj, [src] + hdrs):
            _run([NVCC] + NVFLAGS + (extra_nvflags or []) + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    for s in CPP_SOURCES:
        src, obj = os.path.join(CSRC, s), os.path.join(BUILD, s + ".o")
        if _stale(obj, [src] + hdrs):
            _run(["g++"] + CXXFLAGS + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lz", "-lpthread"], verbose)
    main_src, main_obj = os.path.join(CSRC, "galn_main.cpp"), os.path.join(BUILD, "galn_main.cpp.o")
    if _stale(main_obj, [main_src] + hdrs):
        _run(["g++"] + CXXFLAGS + ["-c", main_src, "-o", main_obj], verbose)
    if _stale(CLI, [main_obj, LIB]):
        _run(["g++", "-o", CLI, main_obj, "-L" + HERE, "-lgalnb200", "-Wl,-rpath,$ORIGIN/..",
              "-L" + os.path.join(CUDA, "lib64"), "-lcudart", "-lpthread"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
