"""Build recipe for libclaw2.so, the sm_100a CUDA library behind pyclaw_b200.

    python -m pyclaw_b200.build          # or pyclaw_b200.build.build()

Compiles csrc/claw2_capi.cu (which includes the tile kernels and Riemann
solvers) with nvcc for sm_100a only, without FMA contraction so that the step
keeps the reference's rounding, into pyclaw_b200/libclaw2.so (in-tree, so the
library travels with the source tree).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libclaw2.so")
SRC = os.path.join(HERE, "csrc", "claw2_capi.cu")
DEPS = [SRC,
        os.path.join(HERE, "csrc", "claw2_kernels.cuh"),
        os.path.join(HERE, "csrc", "claw2_riemann.cuh"),
        os.path.join(ROOT, "include", "claw2.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared", "-cudart", "shared",
]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: cannot build libclaw2.so")


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in DEPS if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    """Compile libclaw2.so if it is missing or older than its sources."""
    if not force and not stale():
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc_path()] + NVCC_FLAGS + list(extra) + ["-o", tmp, SRC]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else ())
