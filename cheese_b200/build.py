"""Build the sm_100a library and the drop-in binaries in-tree (nvcc cross-compiles without a GPU).

    python -m cheese_b200.build [--force] [--verbose]

Outputs (git-ignored, carried to the GPU host with the working tree):
    cheese_b200/lib/libcheese_b200.so     the C ABI of include/cheese_b200.h
    cheese_b200/bin/cheese                drop-in for the reference's build/cheese
    cheese_b200/bin/tcount                drop-in for the reference's build/tcount
    cheese_b200/bin/cliffopt              drop-in for the reference's build/cliffopt
    cheese_b200/bin/rus                   drop-in for the reference's build/rus
    cheese_b200/bin/cheese-spec           the reference's spec writers (spec.py, tcount.py spec) as one binary
"""
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib" / "libcheese_b200.so"
BIN = PKG / "bin"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = os.environ.get("CZ_HOSTCXX", "/usr/bin/g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-ccbin", HOSTCXX, "-Xcompiler", "-fPIC"]

LIB_SOURCES = ["cz_search.cu", "cz_tcount.cu", "cz_clifford.cu", "cz_rus.cu", "cz_spec.cpp", "cz_specgen.cpp",
               "cz_capi.cpp", "cz_serve.cpp"]
HEADERS = ["cz_common.h", "cz_spec.h", "cz_engine.h", "cz_sort.cuh", "cz_tcount.h", "cz_clifford.h", "cz_tableau.h",
           "cz_capi_internal.h", "cz_specgen.h", "cz_rus.h", "cz_rus_node.h"]
BINARIES = {"cheese": "cli_cheese.cpp", "tcount": "cli_tcount.cpp", "cliffopt": "cli_cliffopt.cpp",
            "cheese-spec": "cli_spec.cpp", "rus": "cli_rus.cpp"}


def _stale(out, deps):
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(map(str, cmd)), file=sys.stderr)
    p = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if p.returncode:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError(f"build failed: {' '.join(map(str, cmd[:3]))} ...")
    if verbose and (p.stdout or p.stderr):
        sys.stderr.write(p.stdout + p.stderr)


def build(force=False, verbose=False, ptxas_info=False):
    deps = [CSRC / s for s in LIB_SOURCES + HEADERS] + [ROOT / "include" / "cheese_b200.h"]
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    if force or _stale(LIB, deps):
        objs = []
        for s in LIB_SOURCES:
            o = objdir / (s + ".o")
            extra = ["-Xptxas", "-v"] if (ptxas_info and s.endswith(".cu")) else []
            _run([NVCC, *COMMON, *ARCH, *extra, "-c", CSRC / s, "-o", o], verbose or ptxas_info)
            objs.append(o)
        _run([NVCC, *COMMON, *ARCH, "-shared", *objs, "-o", LIB, "-lcudart", "-lpthread"], verbose)
    for name, src in BINARIES.items():
        out = BIN / name
        if force or _stale(out, [CSRC / src, LIB, ROOT / "include" / "cheese_b200.h"]):
            _run([HOSTCXX, "-std=c++17", "-O2", CSRC / src, "-o", out, f"-L{LIB.parent}", "-lcheese_b200",
                  "-Wl,-rpath,$ORIGIN/../lib", "-L/usr/local/cuda/lib64", "-lcudart"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
