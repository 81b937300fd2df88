"""Build libhbdia_b200.so in-tree (hbdia_b200/libhbdia_b200.so).

CUDA sources are compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a -lineinfo``); host sources with the
system C++ compiler and OpenMP.  The CUDA runtime is linked statically so the
library does not depend on which libcudart.so is first on the loader path;
it shares the device's primary context with any other CUDA user in the
process (PyTorch included), so device pointers and streams interoperate.

Run ``python -m hbdia_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libhbdia_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["plan.cu", "autotune.cu", "cg.cu", "noalloc.cu", "batch.cu", "convert_gpu.cu", "halo.cu", "layout_plan.cu"]
CPP_SOURCES = ["convert.cpp", "generate.cpp", "capi.cpp", "hbdia_cxx.cpp", "serve.cpp", "dia.cpp", "partition.cpp"]
HEADERS = ["hbdia_internal.hpp", "spmv_kernels.cuh", "spmv_xstage.cuh", "spmv_quad.cuh", "spmm_kernels.cuh", "args.cuh",
           "batch_kernels.cuh", "handles.hpp"]


# the C++ drop-in headers, in the reference's include/ shape
CXX_HEADERS = ["Format/HBDIA.hpp", "Format/HBDIAVector.hpp", "Operations/HBDIASpMV.hpp", "types.hpp"]


def _cxx() -> str:
    return os.environ.get("CXX") or shutil.which("g++") or "g++"


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}):\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout.strip() or r.stderr.strip()):
        print(r.stdout + r.stderr, flush=True)
    return r


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "hbdia_b200.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs) or ptxas_info:
            cmd = [NVCC, "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
                   "--expt-relaxed-constexpr", *inc, "-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd, verbose or ptxas_info)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs + [os.path.join(ROOT, "include", "hbdia", h) for h in CXX_HEADERS]):
            _run([_cxx(), "-std=c++17", "-O3", "-fPIC", "-fopenmp", "-Wall", *inc,
                  "-I", os.path.join(CUDA_HOME, "include"), "-c", s, "-o", o], verbose)
    if _stale(LIB, objs):
        # libstdc++ and libgomp by soname: some compiler wrappers cannot link
        # with -fopenmp and would otherwise pull in a static libstdc++.
        _run([_cxx(), "-shared", "-o", LIB, *objs, "-L", os.path.join(CUDA_HOME, "lib64"),
              "-l:libcudart_static.a", "-ldl", "-lrt", "-lpthread",
              "-l:libstdc++.so.6", "-l:libgomp.so.1", "-Wl,--no-undefined"], verbose)
    build_cpp_tests(verbose)
    return LIB


CPP_TEST_SRC = os.path.join(ROOT, "tests", "cpp", "test_dropin.cpp")
CPP_TEST_BIN = os.path.join(BUILD, "test_dropin")


def build_cpp_tests(verbose: bool = False) -> str:
    """The C++ drop-in test program (tests/cpp/test_dropin.cpp), linked
    against the in-tree library."""
    deps = [CPP_TEST_SRC, LIB] + [os.path.join(ROOT, "include", "hbdia", h) for h in CXX_HEADERS]
    if os.path.exists(CPP_TEST_SRC) and _stale(CPP_TEST_BIN, deps):
        _run([_cxx(), "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
              "-I", os.path.join(CUDA_HOME, "include"), CPP_TEST_SRC, "-o", CPP_TEST_BIN, LIB,
              "-Wl,-rpath,$ORIGIN/..", "-L", os.path.join(CUDA_HOME, "lib64"),
              "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64"), "-lcudart", "-l:libstdc++.so.6"], verbose)
    return CPP_TEST_BIN


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
