"""Build recipe of the CUDA library (librtnn_b200.so) and the optixNSearch CLI.

Compiles every .cu of rtnn_b200/csrc for sm_100a with nvcc and links them into
rtnn_b200/lib/librtnn_b200.so (static cudart, C ABI of include/rtnn.h). The CLI
rtnn_b200/bin/optixNSearch links against that library. Incremental: a target is rebuilt
only when one of its sources or headers is newer. Stands in for the reference's CMake build
of optixNSearch (src/optixNSearch/CMakeLists.txt); its compile-time KNN K (-DKNN, lines
58-61) becomes the CLI's -DRTNN_KNN default, while the library takes K at run time.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIBDIR = os.path.join(HERE, "lib")
BINDIR = os.path.join(HERE, "bin")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "librtnn_b200.so")
CLI = os.path.join(BINDIR, "optixNSearch")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
           "-Xptxas", "-O3", "-I" + INCLUDE, "-I" + CSRC]
SOURCES = ["scan.cu", "radix_sort.cu", "build_grid.cu", "search.cu", "partition.cu", "api.cu",
           "noalloc.cu"]


def _headers():
    out = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:4]) + " ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(verbose=False, ptxas_verbose=False):
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BINDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = _headers()
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + hdrs) or ptxas_verbose:
            extra = ["-Xptxas", "-v"] if ptxas_verbose else []
            _run([NVCC] + ARCH + NVFLAGS + extra + ["-c", s, "-o", o], verbose or ptxas_verbose)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs +
             ["-Xlinker", "--no-undefined", "-Xlinker", "-z,defs"], verbose)
    cli_srcs = [os.path.join(CSRC, f) for f in ("cli.cpp", "pointio.cpp")]
    if _stale(CLI, cli_srcs + [LIB, os.path.join(CSRC, "pointio.h")] + hdrs):
        _run(["g++", "-O2", "-std=c++17", "-pthread", "-I" + INCLUDE] + cli_srcs +
             ["-o", CLI, "-L" + LIBDIR, "-lrtnn_b200", "-Wl,-rpath,$ORIGIN/../lib"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
