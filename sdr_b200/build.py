"""Build libsdr_gpu.so in-tree with nvcc for sm_100a (B200).

    python -m sdr_b200.build            # compile if sources changed
    python -m sdr_b200.build --force

The library is a plain C ABI (include/sdr_gpu.h); Python loads it via ctypes.
Host and device code are compiled without FMA contraction (-ffp-contract=off,
--fmad=false): the f64 emission math and the CFL arithmetic follow the
reference's operation order, and every device float operation is rounded on
its own, so a kernel body gives the same bits in every kernel it is inlined
into (a scene's substep alone and inside a packed launch).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsdr_gpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) + glob.glob(os.path.join(HERE, "csrc", "*.cpp")))


def deps():
    return sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(ROOT, "include", "sdr_gpu.h")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--fmad=false", "-shared", "-Xcompiler",
           "-fPIC,-ffp-contract=off",
           "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp", *sources(), "-lz"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
