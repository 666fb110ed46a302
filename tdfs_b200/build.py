"""Build libtdfs_b200.so and the ulb/lb drivers in-tree for sm_100a.

    python -m tdfs_b200.build        (or tdfs_b200.build.build())

Outputs: tdfs_b200/lib/libtdfs_b200.so, tdfs_b200/bin/ulb, tdfs_b200/bin/lb, and
tdfs_b200/bin/tdfs_convert (the host-only graph writer and converter: no CUDA
runtime, so processes that only prepare graph files never load the engine).
nvcc cross-compiles without a GPU; the objects are rebuilt only when a source
is newer than its output.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BINDIR = os.path.join(HERE, "bin")
OBJDIR = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(LIBDIR, "libtdfs_b200.so")
NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O3,-Wall", "--expt-relaxed-constexpr"]

SOURCES = ["error.cpp", "plan.cpp", "csr.cpp", "capi.cpp", "serve.cpp", "graph.cu", "match.cu", "static_count.cu", "estimate.cpp"]
HEADERS = ["common.h", "plan.h", "csr.h", "graph.h", "match.cuh", "serve.h"]


def _newer(src_paths, out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(p) > t for p in src_paths)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(BINDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "tdfs.h")]
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OBJDIR, s + ".o")
        objs.append(obj)
        if _newer([src] + hdrs, obj):
            extra = ["-Xptxas", "-v"] if (ptxas_info and s.endswith(".cu")) else []
            _run([NVCC, *ARCH, *COMMON, *extra, "-c", src, "-o", obj], verbose)
    if _newer(objs, LIB):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"], verbose)
    cli = os.path.join(CSRC, "cli.cpp")
    for name, lab in (("ulb", 0), ("lb", 1)):
        out = os.path.join(BINDIR, name)
        if _newer([cli, LIB], out):
            _run([NVCC, *ARCH, "-std=c++17", "-O2", f"-DTDFS_LABELED={lab}", cli, "-o", out,
                  f"-L{LIBDIR}", "-ltdfs_b200", f"-Xlinker=-rpath,$ORIGIN/../lib"], verbose)
    conv = os.path.join(BINDIR, "tdfs_convert")
    conv_src = [os.path.join(CSRC, s) for s in ("convert.cpp", "csr.cpp", "error.cpp")]
    if _newer(conv_src + hdrs, conv):
        _run([CXX, "-std=c++17", "-O3", "-Wall", "-pthread", *conv_src, "-o", conv], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
