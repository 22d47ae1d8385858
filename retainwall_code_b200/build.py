"""Build the in-tree native library (librw.so, sm_100a) and the `loquat` CLI with nvcc.

    python -m retainwall_code_b200.build [-v]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "librw.so")
CLI = os.path.join(PKG, "loquat")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH
SOURCES = ["rw_engine.cu", "rw_io.cpp", "rw_noalloc.cu", "rw_mlp.cu"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    nvcc = _nvcc()
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "retainwall.h")]
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    if force or _stale(LIB, deps):
        objs = [os.path.join(objdir, os.path.splitext(s)[0] + ".o") for s in SOURCES]
        with ThreadPoolExecutor(len(SOURCES)) as ex:
            list(ex.map(lambda so: _run([nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, so[0]), "-o", so[1]], verbose),
                        zip(SOURCES, objs)))
        _run([nvcc, *ARCH, "-shared", *objs, "-o", LIB], verbose)
    if force or _stale(CLI, deps + [LIB]):
        _run([nvcc, "-std=c++17", "-O2", *ARCH, os.path.join(CSRC, "main.cpp"), "-o", CLI, "-L" + PKG, "-lrw",
              "-Xlinker", "-rpath=$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
