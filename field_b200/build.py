"""Build libsfgpu.so in-tree for sm_100a (B200) with nvcc.

The library is compiled without FMA contraction (``-fmad=false``) so the
propagator arithmetic rounds like SFbox's separate multiply/add CPU loops.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsfgpu.so")
SOURCES = ["sfgpu_system.cu", "sfgpu_solve.cu", "sfgpu_batch.cu", "sfgpu_tangent.cu", "sfgpu_adjoint.cu",
           "sfgpu_noalloc.cu", "sfgpu_newton.cu", "sfgpu_batch_wide.cu"]
HEADERS = ["sfgpu_internal.cuh", "sfgpu_kernels.cuh", "sfgpu_system.h", "sfgpu_batch.cuh", "sfgpu_tangent.cuh",
           "sfgpu_adjoint.cuh", "sfgpu_newton.h", "sfgpu_charge.cuh", "sfgpu_batch_kernel.cuh",
           "../../include/sfgpu.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = _sources() + [os.path.join(CSRC, h) for h in HEADERS]
    deps += glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-fmad=false",
           "-Xcompiler", "-fPIC", "-shared", "-o", LIB + ".tmp", *_sources()]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
