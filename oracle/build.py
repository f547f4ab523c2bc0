"""Build recipe for the CPU oracle (test infrastructure only).

Compiles claw2_oracle.c into two shared libraries next to this file:

  liboracle_claw2.so      -O2 -ffp-contract=off: strict IEEE double, no FMA
                          contraction.  This is the parity build every test
                          compares against.
  liboracle_claw2_omp.so  the same source with -O3 -fopenmp and still
                          -ffp-contract=off, used only to time the CPU baseline
                          on all host cores (results are bit-identical to the
                          parity build; the tests check that).  No -march flag,
                          so the library runs on any x86-64 host it travels to.

Run as ``python oracle/build.py`` or call ``build()``.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "claw2_oracle.c")
LIB = os.path.join(HERE, "liboracle_claw2.so")
LIB_OMP = os.path.join(HERE, "liboracle_claw2_omp.so")

COMMON = ["-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math", "-Wall",
          "-Wno-unused-parameter", "-Wno-unknown-pragmas", "-std=gnu11"]


def _stale(out):
    if not os.path.exists(out):
        return True
    deps = [SRC, os.path.join(HERE, "..", "include", "claw2.h"), __file__]
    return any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile both oracle libraries if missing or stale; return their paths."""
    jobs = [
        (LIB, ["gcc", "-O2"] + COMMON + ["-o", LIB, SRC, "-lm"]),
        (LIB_OMP, ["gcc", "-O3", "-fopenmp", "-DORC_OPENMP"] + COMMON
         + ["-o", LIB_OMP, SRC, "-lm"]),
    ]
    for out, cmd in jobs:
        if force or _stale(out):
            if verbose:
                print(" ".join(cmd))
            tmp = out + ".tmp"
            cmd = [c if c != out else tmp for c in cmd]
            subprocess.run(cmd, check=True)
            os.replace(tmp, out)
    return LIB, LIB_OMP


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
