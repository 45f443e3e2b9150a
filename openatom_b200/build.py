"""Build liboa_gpu.so (sm_100a) in-tree with nvcc.

    python -m openatom_b200.build [--verbose]

The library is a plain C ABI (include/oa_gpu.h); Python loads it with ctypes.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liboa_gpu.so")
SOURCES = ["oa_state.cu", "oa_pencil.cu", "oa_pair_plane.cu", "oa_rho.cu", "oa_rho_pencil.cu", "oa_pc.cu", "oa_dgemm.cu", "oa_ns.cu", "oa_umma.cu", "oa_tgemm.cu", "oa_ozaki.cu", "oa_nl.cu", "oa_ions.cu", "oa_eesl.cu", "oa_step.cu", "oa_noalloc.cu", "oa_abi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(verbose: bool = False, force: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "oa_gpu.h"))
    if not force and os.path.exists(LIB):
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-rdc=false",
                    "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    if verbose:
        flags += ["-Xptxas", "-v"]
    for s in srcs:
        o = os.path.join(objdir, os.path.basename(s) + ".o")
        cmd = [nvcc()] + flags + ["-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"nvcc failed on {s}")
        objs.append(o)
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
