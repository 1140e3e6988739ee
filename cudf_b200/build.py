"""Builds the engine's shared library in-tree: cudf_b200/_build/libcudf_b200.so.

nvcc cross-compiles for sm_100a (B200); no GPU is needed to build.
Usage: python -m cudf_b200.build [--verbose]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libcudf_b200.so")

SOURCES = ["gb_engine.cu", "gb_sorted.cu", "gb_scatter.cu", "gb_capi.cu", "gb_noalloc.cu", "gb_batch.cu", "gb_server.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _deps_newer(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".h", ".hpp")) and os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    hdr = os.path.join(ROOT, "include", "cudf_b200.h")
    return os.path.getmtime(hdr) > t


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    objs = []

    def compile_one(s):
        src = os.path.join(CSRC, s)
        obj = os.path.join(OUT, s.replace(".cu", ".o"))
        if force or _deps_newer(obj, src):
            cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {s}:\n{r.stdout}\n{r.stderr}")
            if verbose and r.stderr:
                print(r.stderr, flush=True)
        return obj

    with cf.ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        objs = list(ex.map(compile_one, srcs))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


CPP_TESTS = os.path.join(ROOT, "tests", "cpp")
CPP_TEST_BIN = os.path.join(OUT, "groupby_api_golden")


def build_cpp_tests() -> str:
    """Compiles the C++ program that drives the engine through
    include/cudf_b200/groupby.hpp (libcudf's groupby API shapes), linked
    against the in-tree library; used by tests/test_gpu_cpp_api.py."""
    lib = build()
    src = os.path.join(CPP_TESTS, "groupby_api_golden.cpp")
    hdrs = [os.path.join(ROOT, "include", "cudf_b200", "groupby.hpp"), os.path.join(ROOT, "include", "cudf_b200.h")]
    if (os.path.exists(CPP_TEST_BIN) and all(os.path.getmtime(CPP_TEST_BIN) > os.path.getmtime(f)
                                             for f in [src, lib, *hdrs])):
        return CPP_TEST_BIN
    cuda = os.path.dirname(os.path.dirname(NVCC))
    cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(cuda, "include"), src, "-o", CPP_TEST_BIN, "-L", OUT, "-lcudf_b200",
           "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"C++ API test build failed:\n{r.stdout}\n{r.stderr}")
    return CPP_TEST_BIN


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
    print(build_cpp_tests())
