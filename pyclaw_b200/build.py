"""Build recipe for libclaw2.so, the sm_100a CUDA library behind pyclaw_b200.

    python -m pyclaw_b200.build          # or pyclaw_b200.build.build()

Compiles csrc/claw2_capi.cu (the plain and batched steps, which include the
tile kernels and Riemann solvers) and csrc/claw2_adjoint.cu (multi-shot
acoustics and its adjoint) with nvcc for sm_100a only, without FMA contraction
so that the step keeps the reference's rounding, as two objects compiled in
parallel under pyclaw_b200/_build/, and links them into pyclaw_b200/libclaw2.so
(in-tree, so the library travels with the source tree).
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libclaw2.so")
SRCS = [os.path.join(HERE, "csrc", "claw2_capi.cu"),
        os.path.join(HERE, "csrc", "claw2_adjoint.cu")]
OBJDIR = os.path.join(HERE, "_build")
DEPS = SRCS + [os.path.join(HERE, "csrc", "claw2_kernels.cuh"),
               os.path.join(HERE, "csrc", "claw2_devattr.h"),
               os.path.join(HERE, "csrc", "claw2_riemann.cuh"),
               os.path.join(HERE, "csrc", "claw2_light.cuh"),
               os.path.join(HERE, "csrc", "claw2_lean.cuh"),
               os.path.join(HERE, "csrc", "claw2_tma.cuh"),
               os.path.join(ROOT, "include", "claw2.h"),
               os.path.join(ROOT, "include", "claw2_adjoint.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
]
LINK_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-cudart", "shared"]


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
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = nvcc_path()
    procs = []
    objs = []
    for src in SRCS:
        obj = os.path.join(OBJDIR, os.path.splitext(os.path.basename(src))[0] + ".o")
        cmd = [nvcc] + NVCC_FLAGS + list(extra) + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd), cmd))
        objs.append(obj)
    failed = [cmd for p, cmd in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    tmp = LIB + ".tmp"
    cmd = [nvcc] + LINK_FLAGS + ["-o", tmp] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else ())
