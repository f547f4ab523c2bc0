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

A third library is only ever built on the machine that times the CPU
baseline, by ``build_timing()``:

  liboracle_claw2_native_<key>.so  -O3 -march=native -fopenmp with the compiler's
                          default floating-point contraction (FMA allowed):
                          the fastest build of the same source for this host,
                          used for timing only, never for parity.  <key> is a
                          hash of the host's CPU model and feature flags and of
                          the compiler, so a copy built on another machine is
                          never loaded here.

Run as ``python oracle/build.py`` or call ``build()``.
"""
import hashlib
import os
import platform
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


TIMING_FLAGS = ["-O3", "-march=native", "-fopenmp", "-DORC_OPENMP", "-fPIC", "-shared", "-fno-fast-math",
                "-std=gnu11", "-w"]


def host_cpu():
    """(model name, feature-flags line) of this host's first CPU."""
    model, flags = platform.processor() or "unknown", ""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name") and model in ("unknown", "x86_64", ""):
                    model = ln.split(":", 1)[1].strip()
                elif ln.startswith("flags") and not flags:
                    flags = ln.split(":", 1)[1].strip()
                if flags and model not in ("unknown", "x86_64", ""):
                    break
    except OSError:
        pass
    return model, flags


def build_timing(verbose=False):
    """Compile (if needed) the host-native timing build; returns (path, flags, cpu model)."""
    model, flags = host_cpu()
    try:
        cc = subprocess.run(["gcc", "--version"], capture_output=True, text=True).stdout.splitlines()[0]
    except (OSError, IndexError):
        cc = "gcc"
    key = hashlib.sha1(("%s|%s|%s|%s" % (model, flags, cc, " ".join(TIMING_FLAGS))).encode()).hexdigest()[:12]
    out = os.path.join(HERE, "liboracle_claw2_native_%s.so" % key)
    if _stale(out):
        cmd = ["gcc"] + TIMING_FLAGS + ["-o", out + ".tmp", SRC, "-lm"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(out + ".tmp", out)
    return out, "gcc " + " ".join(TIMING_FLAGS) + " (" + cc + ")", model


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
