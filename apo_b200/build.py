"""Build recipe of the CUDA library (apo_b200/libapo2.so), compiled in-tree for sm_100a.

The kernels are compiled with --use_fast_math, the floating-point mode of the reference
library's CUDA code, so that single-precision traversal decisions are taken on the same
values; double precision is not affected by that flag.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libapo2.so")
SOURCES = ["sort.cu", "lbvh.cu", "cells.cu", "speculate.cu", "certify.cu", "cavity.cu", "api.cu", "sort_static.cu", "calibrate.cu", "proposal.cu", "generators.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--use_fast_math", "-Xcompiler", "-fPIC,-O2",
         "-I", os.path.join(ROOT, "include")]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    built = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "apo2.h")]
    return any(os.path.getmtime(d) > built for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compiles every .cu source and links libapo2.so; returns its path."""
    if not force and not _stale():
        return LIB
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    nvcc = _nvcc()
    objects = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(obj_dir, src + ".o")
        if src.endswith(".cpp"):
            cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-I", os.path.join(ROOT, "include"), "-c",
                   os.path.join(CSRC, src), "-o", obj]
        else:
            cmd = [nvcc, *ARCH, *FLAGS, *(extra or []), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objects.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append(f"{src}:\n{out}")
        elif verbose and out.strip():
            print(out, file=sys.stderr)
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(failed))
    tmp = LIB + ".tmp"
    subprocess.run([nvcc, *ARCH, "-shared", *objects, "-o", tmp, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a.startswith("-X")])
    print(LIB)
