"""Build the in-tree shared library ``hermes3d_b200/libh3dg.so``.

Host C++ (mesh, space, plan) is compiled with g++; the CUDA sources are
compiled by nvcc for sm_100a only.  The library is written next to this
file so it travels with the source tree.

    python -m hermes3d_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libh3dg.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SRC = ["host/h3dg_host.cpp"]
CUDA_SRC = ["h3dg_capi.cu", "tables_lo.cu", "tables_seg.cu", "tables_lo_tc.cu", "tables_stock.cu", "tables_ho.cu", "tables_ho_tc.cu", "tables_adj.cu", "tables_mixed.cu", "tables_ho_oz.cu", "tables_dm.cu"]


def _deps():
    out = []
    for d, _, files in os.walk(CSRC):
        out += [os.path.join(d, f) for f in files if f.endswith((".h", ".cuh", ".cu", ".cpp"))]
    out.append(os.path.join(ROOT, "include", "h3dg.h"))
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
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    deps = _deps()
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    jobs = []
    objs = []
    for s in HOST_SRC:
        o = os.path.join(OBJDIR, os.path.basename(s) + ".o")
        objs.append(o)
        jobs.append([CXX, "-O3", "-std=c++17", "-fPIC", "-pthread", "-Wall", *inc, "-c", os.path.join(CSRC, s), "-o", o])
    for s in CUDA_SRC:
        o = os.path.join(OBJDIR, os.path.basename(s) + ".o")
        objs.append(o)
        jobs.append([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", *inc, "-c", os.path.join(CSRC, s), "-o", o])
    with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lpthread"], verbose)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    sys.exit(0)
