"""Builds libpsg.so (the CUDA hot path + its C ABI) in-tree for sm_100a.

    python -m psphray_b200.build [--force]

Every translation unit is compiled without floating-point contraction
(-fmad=false on the device, -ffp-contract=off on the host) so that products
and sums round once each, in the order written, as the reference's x86 code
does; the geometric accept/reject decisions depend on it.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpsg.so")
RUN = os.path.join(HERE, "psg_run")

CU_SOURCES = ["psg_context.cu", "psg_tree.cu", "psg_trace.cu", "psg_tick.cu", "psg_emit.cu", "psg_mlp.cu", "psg_surrogate.cu",
              "psg_recomb.cu"]
C_SOURCES = ["psg_host.c", "psg_snapshot.c"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h")))

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I", INCLUDE, "-I", CSRC, "--expt-relaxed-constexpr"] + ARCH


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[-1]}")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "psg.h"), __file__]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
        objs.append(o)
    for src in C_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".c", ".o"))
        if force or _stale(o, [s] + hdrs):
            _run(["gcc", "-O2", "-std=gnu11", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
                  "-I", INCLUDE, "-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    # the C host driver over the library's C ABI
    src = os.path.join(CSRC, "psg_run.c")
    if force or _stale(RUN, [src, LIB, os.path.join(INCLUDE, "psg.h")]):
        _run(["gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-I", INCLUDE, src, "-L", HERE, "-lpsg",
              "-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,$ORIGIN", "-lm", "-o", RUN])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
