"""Builds libtenrso_b200.so in-tree with nvcc for sm_100a only.

Usage: python -m tenrso_b200.build [--force]
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libtenrso_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-O3",
    "-I", os.path.join(ROOT, "include"),
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _shared_deps():
    """Files every translation unit depends on (headers and the flags here)."""
    return glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(ROOT, "include", "tenrso_b200.h"), __file__]


def _newer(path: str, deps) -> bool:
    if not os.path.exists(path):
        return True
    t = os.path.getmtime(path)
    return any(os.path.getmtime(d) > t for d in deps)


def _stale() -> bool:
    return _newer(LIB, sources() + _shared_deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    shared = _shared_deps()
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        # an object is rebuilt when its source, a shared header or these
        # flags changed since it was compiled
        if not (force or verbose) and not _newer(obj, [src] + shared):
            continue
        cmd = [NVCC, *FLAGS, "-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT)))
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out.decode())
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"nvcc failed on {src}\n")
    if failed:
        raise RuntimeError("nvcc build failed")
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                    "-o", tmp, *objs, "-cudart", "static", "-lpthread", "-ldl", "-lrt"],
                   check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
