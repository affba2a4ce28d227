"""Build the sm_100a shared library ``phlegethon_b200/_lib/libphl_b200.so`` in-tree.

The FP64 unit is compiled with ``--fmad=false``: the reference's CPU build targets baseline
x86-64 (no FMA, Make.local/Make.pkgconfig:91-93), and keeping every multiply and add separately
rounded lets the FP64 path reproduce it bit for bit.  The FP32 split-precision unit is compiled
with contraction on and approximate FP32 division/square root.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
BUILDDIR = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libphl_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# (source, extra flags)
UNITS = [
    ("phl_runtime.cu", ["--fmad=false"]),
    # FP32 flux arithmetic of the split form: approximate (2 ulp) division and square root,
    # FP32 denormals flushed; the FP64 EoS/state arithmetic in this unit is unaffected
    ("phl_split.cu", ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources_newer(target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    for root in (CSRC, os.path.join(HERE, "..", "include")):
        for f in os.listdir(root):
            if f.endswith((".cu", ".cuh", ".h")) and os.path.getmtime(os.path.join(root, f)) > t:
                return True
    return False


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every CUDA unit for sm_100a and link the shared library; return its path."""
    if not force and not _sources_newer(LIB):
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILDDIR, exist_ok=True)
    nvcc = _nvcc()
    objs, procs = [], []
    # the units are independent: compile them concurrently
    for src, extra in UNITS:
        obj = os.path.join(BUILDDIR, src.replace(".cu", ".o"))
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-rdc=false",
               "-Xptxas", "-warn-spills", *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd)))
        objs.append(obj)
    failed = [src for src, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(failed))
    tmp = LIB + ".tmp"
    subprocess.run([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
