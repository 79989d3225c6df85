"""Build ``gpu_b200/libctrecon.so`` from ``gpu_b200/csrc`` with nvcc for sm_100a.

Object files go to ``gpu_b200/_build``; the shared library is written in-tree
next to this file, statically linked against the CUDA runtime so that it does
not depend on which libcudart another module in the process loaded first.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libctrecon.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-I", INCLUDE, "-I", SRC]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def _sources():
    return sorted(f for f in os.listdir(SRC) if f.endswith((".cu", ".cpp")))


def _deps_mtime():
    files = [os.path.join(SRC, f) for f in os.listdir(SRC)]
    files.append(os.path.join(INCLUDE, "ctrecon.h"))
    return max(os.path.getmtime(f) for f in files)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compile every source (in parallel, one nvcc per source) and link the
    library; returns its path."""
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(OUT_DIR, exist_ok=True)
    deps = _deps_mtime()
    objs, cmds = [], []
    for f in _sources():
        src = os.path.join(SRC, f)
        obj = os.path.join(OUT_DIR, f + ".o")
        objs.append(obj)
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= deps:
            continue
        cmd = [nvcc(), *ARCH, *NVFLAGS, "-c", src, "-o", obj]
        if ptxas_verbose and f.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        cmds.append(cmd)
    workers = max(1, min(len(cmds), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        for r in list(pool.map(lambda c: subprocess.run(c), cmds)):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas" in sys.argv)
    print(LIB)
