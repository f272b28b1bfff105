"""Build libket_b200.so in-tree (sm_100a only).

``python ket_b200/build.py`` (or ``__graft_entry__.build()``; not ``-m``, which imports
the package and so the library being rebuilt) compiles every
CUDA source under ket_b200/csrc with nvcc for ``compute_100a/sm_100a`` and the
host sources with g++ (C++20), and links ``ket_b200/libket_b200.so`` with the
CUDA runtime linked statically.  Objects go to ket_b200/_build; a source is
recompiled only when it or a header is newer than its object.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libket_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
CXX = os.environ.get("CXX", "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                  "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + OBJ]
CXXFLAGS = ["-O2", "-std=c++20", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wextra",
            "-I" + os.path.join(CUDA, "include"), "-I" + os.path.join(ROOT, "include")]


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(src, obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def _embed_tile_source():
    """adj_tile.cuh as a C++ string literal (the per-block adjoint kernels are
    compiled from it at run time)."""
    src = os.path.join(CSRC, "adj_tile.cuh")
    out = os.path.join(OBJ, "adj_tile_src.inc")
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    text = open(src).read()
    assert ')KBSRC"' not in text
    with open(out, "w") as f:
        f.write('R"KBSRC(' + text + ')KBSRC"\n')
    return out


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    deps = _headers() + [_embed_tile_source()]
    objs, jobs = [], []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(src, obj, deps) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + NVFLAGS + extra + ["-c", src, "-o", obj])
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(src, obj, deps):
            jobs.append([CXX] + CXXFLAGS + ["-c", src, "-o", obj])
    # compile in parallel
    procs = []
    for cmd in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or (ptxas_info and out):
            sys.stderr.write(out)
        if p.returncode != 0:
            failed = True
            # make sure a stale object is not reused
            try:
                os.remove(cmd[cmd.index("-o") + 1])
            except (OSError, ValueError):
                pass
    if failed:
        raise RuntimeError("ket_b200: compilation failed")
    if jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs +
             ["-Xcompiler", "-fPIC", "-Xlinker", "--no-undefined", "-lpthread", "-ldl"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
