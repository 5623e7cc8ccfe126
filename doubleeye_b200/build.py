"""Build the in-tree CUDA library (sm_100a) with nvcc.

    python -m doubleeye_b200.build           # builds doubleeye_b200/_lib/libdoubleeye_b200.so

The library is built in place so it travels with the source tree; nothing is
installed into site-packages and there is no JIT cache.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(OUT_DIR, "libdoubleeye_b200.so")

SOURCES = ["de_dense.cu", "de_capi.cu", "de_noalloc.cu", "de_sparse.cu", "de_edges.cu",
           "de_serve.cu", "de_graph.cu", "de_prior.cu", "de_fill.cu"]
# the bench's integer-pipe probe: its own library, outside the matcher's C ABI
PROBE_SRC = "de_probe.cu"
PROBE_LIB = os.path.join(OUT_DIR, "libde_probe.so")
TOOLS = os.path.join(PKG, "tools")
CLI = os.path.join(OUT_DIR, "de_dense_gpu")      # the reference-compatible command line
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # the row solve's float arithmetic must not be contracted into FMAs: it is
    # compared bit for bit with the reference's x86-64 single precision
    "--fmad=false",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-O2",
    "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build")


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _stamp() -> str:
    return " ".join(NVCC_FLAGS + [os.path.basename(s) for s in sources()])


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    stamp = LIB + ".cmd"
    if not os.path.exists(stamp) or open(stamp).read() != _stamp():
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f != PROBE_SRC]
    deps.append(os.path.join(os.path.dirname(PKG), "include", "doubleeye_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_cli(force: bool = False, verbose: bool = False) -> str:
    """de_dense_gpu: a host-only C++ program over the C ABI (g++, rpath to the lib)."""
    src = os.path.join(TOOLS, "de_dense_gpu.cpp")
    hdr = os.path.join(os.path.dirname(PKG), "include", "doubleeye_b200.h")
    if (not force and os.path.exists(CLI) and
            os.path.getmtime(CLI) >= max(os.path.getmtime(src), os.path.getmtime(hdr),
                                         os.path.getmtime(LIB))):
        return CLI
    cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-Wall",
           "-I", os.path.dirname(hdr), src, "-L", OUT_DIR, "-ldoubleeye_b200",
           "-Wl,-rpath,$ORIGIN", "-o", CLI + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(CLI + ".tmp", CLI)
    return CLI


def build_probe(force: bool = False, verbose: bool = False) -> str:
    src = os.path.join(CSRC, PROBE_SRC)
    if not force and os.path.exists(PROBE_LIB) and \
            os.path.getmtime(PROBE_LIB) >= os.path.getmtime(src):
        return PROBE_LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", PROBE_LIB + ".tmp", src]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(PROBE_LIB + ".tmp", PROBE_LIB)
    return PROBE_LIB


CPP_SRC = os.path.join(PKG, "cpp", "doubleeye_shim.cpp")
CPP_LIB = os.path.join(OUT_DIR, "libdoubleeye_cpp.a")   # the C++14 surface over the C ABI


def build_cpp(force: bool = False, verbose: bool = False) -> str:
    """libdoubleeye_cpp.a: the reference's C++ call surface (include/doubleeye/*.hpp)
    over the C ABI; callers link it with libdoubleeye_b200.so."""
    inc = os.path.join(os.path.dirname(PKG), "include")
    deps = [CPP_SRC] + [os.path.join(inc, "doubleeye", f) for f in os.listdir(os.path.join(inc, "doubleeye"))]
    deps.append(os.path.join(inc, "doubleeye_b200.h"))
    if not force and os.path.exists(CPP_LIB) and \
            os.path.getmtime(CPP_LIB) >= max(os.path.getmtime(d) for d in deps):
        return CPP_LIB
    obj = CPP_LIB[:-2] + ".o"
    cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++14", "-fPIC", "-Wall", "-I", inc,
           "-c", CPP_SRC, "-o", obj]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    subprocess.run(["ar", "rcs", CPP_LIB + ".tmp", obj], check=True)
    os.replace(CPP_LIB + ".tmp", CPP_LIB)
    return CPP_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    build_probe(force, verbose)
    build_cpp(force, verbose)
    if not force and not stale():
        build_cli(False, verbose)
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", tmp] + sources()
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    with open(LIB + ".cmd", "w") as f:
        f.write(_stamp())
    os.replace(tmp, LIB)
    build_cli(True, verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
