"""Build libpenguin_b200.so in-tree for sm_100a (nvcc, no JIT cache).

    python -m penguin_2_0_b200.build        # or __graft_entry__.build()
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libpenguin_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"]
SOURCES = ["pg_host.cpp", "pg_kernels.cu", "pg_kernels32.cu", "pg_run.cu", "pg_batch.cu", "pg_serve.cpp", "pg_noalloc.cu"]


def _newer(out, deps):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "penguin_b200.h"))
    objs, procs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src + ".o")
        objs.append(o)
        if not force and _newer(o, [s] + headers):
            continue
        cmd = ["nvcc", *ARCH, *NVFLAGS, "-c", s, "-o", o]
        if src.endswith(".cpp"):
            cmd = ["nvcc", "-x", "c++", *NVFLAGS, "-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{out}")
        if verbose and out.strip():
            print(out)
    if force or not _newer(OUT, objs):
        cmd = ["nvcc", *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
