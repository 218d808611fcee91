"""Build libqaf.so (the CUDA kernels + C ABI) into nature-control_b200/qaf/.

    python nature-control_b200/build.py [--force] [--jobs N]

Compiles for sm_100a only (B200) with nvcc; cross-compiles without a GPU.
The library is rebuilt when any source under csrc/ or include/ is newer.
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "qaf", "libqaf.so")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def needs_build(out=OUT):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps())


def build(force=False, verbose=True, extra=()):
    if not force and not needs_build():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    # QAF_SPLIT_COMPILE=1: compile each file's kernels in parallel threads
    # (shorter builds while iterating; timed builds use the default)
    if os.environ.get("QAF_SPLIT_COMPILE") == "1":
        extra = (*extra, "--split-compile=0")
    objs = []
    tmpdir = os.path.join(PKG, "_build")
    os.makedirs(tmpdir, exist_ok=True)
    procs = []
    for src in sources():
        obj = os.path.join(tmpdir, os.path.basename(src) + ".o")
        cmd = [nvcc, *[f for f in NVCC_FLAGS if f != "-shared"], "-c", "-I", os.path.join(ROOT, "include"),
               *extra, "-o", obj, src]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((subprocess.Popen(cmd), src))
        objs.append(obj)
    for p, src in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed on {src}")
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT + ".tmp", *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force))
    sys.exit(0)
