"""Regenerate the golden fixtures in this folder from the reference tree.

The reference's own regression tests compare whole runs against text files
written by an earlier verified run.  This script converts those files, value
for value, into compressed .npz fixtures so that the tests here can use them
without the reference tree being present:

  shockbubble_density.npz   apps/euler_2d/verify_shockbubble_classic.txt
                            (density, 160x40; test_euler2d_shockbubble.py:15-19,
                            abstol 1e-12 on the 2-norm of the difference)
  acoustics_pressure.npz    apps/acoustics_2d_homogeneous/verify_classic.txt
                            (pressure, 100x100; test_2d_acoustics.py:115-116,
                            reltol 1e-3)
  vc_acoustics_pressure.npz apps/acoustics_2d_variable/pressure_classic.txt
                            (pressure, 200x200; test_acoustics_2d_variable.py:111-115,
                            max-abs 0.1)
  vc_acoustics_io.npz       apps/acoustics_2d_variable/io_test_verification/
                            fort.q0020 (q, 3x200x200), fort.a0000 (aux, 2x200x200)
                            and the fort.t headers (test_acoustics_2d_variable_io.py,
                            reltol 1e-4)
  psystem_gauges.npz        apps/psystem_2d/verify_gauge<x>_<y>.txt, the four
                            gauges' (t, p, 10 p) rows (test_2d_psystem.py:9-30,
                            reltol 1e-4)

Usage: python tests/golden/make_golden.py /path/to/reference
   or: CLAW2_REFERENCE=/path/to/reference python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_fort(path, nvar):
    """Parse a Clawpack ascii fort.q / fort.a file (src/pyclaw/io/ascii.py:44-99)."""
    with open(path) as f:
        lines = f.read().splitlines()
    mx = int(lines[2].split()[0])
    my = int(lines[3].split()[0])
    vals = []
    for ln in lines[8:]:
        parts = ln.split()
        if parts:
            vals.extend(float(v) for v in parts)
    a = np.array(vals).reshape(my, mx, nvar)      # written j-major, then i, then m
    return np.ascontiguousarray(np.transpose(a, (2, 1, 0)))   # -> (m, i, j)


PSYSTEM_GAUGES = ("0.25_0.25", "17.85_1.25", "3.25_18.75", "11.75_11.75")


def psystem(ref):
    apps = os.path.join(ref, "apps")
    g = {"g" + k.replace(".", "p"): np.loadtxt(os.path.join(apps, "psystem_2d", "verify_gauge%s.txt" % k))
         for k in PSYSTEM_GAUGES}
    np.savez_compressed(os.path.join(HERE, "psystem_gauges.npz"), **g)


def main(ref):
    psystem(ref)
    apps = os.path.join(ref, "apps")
    d = np.loadtxt(os.path.join(apps, "euler_2d", "verify_shockbubble_classic.txt"))
    np.savez_compressed(os.path.join(HERE, "shockbubble_density.npz"), density=d)
    p = np.loadtxt(os.path.join(apps, "acoustics_2d_homogeneous", "verify_classic.txt"))
    np.savez_compressed(os.path.join(HERE, "acoustics_pressure.npz"), pressure=p)
    p = np.loadtxt(os.path.join(apps, "acoustics_2d_variable", "pressure_classic.txt"))
    np.savez_compressed(os.path.join(HERE, "vc_acoustics_pressure.npz"), pressure=p)
    io = os.path.join(apps, "acoustics_2d_variable", "io_test_verification")
    q20 = read_fort(os.path.join(io, "fort.q0020"), 3)
    a0 = read_fort(os.path.join(io, "fort.a0000"), 2)
    t20 = float(open(os.path.join(io, "fort.t0020")).readline().split()[0])
    with open(os.path.join(io, "fort.t0020")) as f:
        t_header = f.read()
    with open(os.path.join(io, "fort.q0020")) as f:
        q_header = "\n".join(f.read().splitlines()[:8])
    np.savez_compressed(os.path.join(HERE, "vc_acoustics_io.npz"), q20=q20, aux0=a0,
                        t20=t20, t_header=t_header, q_header=q_header)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CLAW2_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py /path/to/reference  (or set CLAW2_REFERENCE)")
    main(ref)
