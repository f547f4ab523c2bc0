"""Clawpack ascii frames (src/pyclaw/io/ascii.py:14-150) written and read by
pyclaw_b200.io.ascii, checked on the host against the reference's own frame
files (apps/acoustics_2d_variable/io_test_verification, stored value for value
in tests/golden/vc_acoustics_io.npz).

The states written here come from the oracle's replay of the variable-
coefficient acoustics app (apps/acoustics_2d_variable/acoustics.py:8-88), so
the file format, the header lines and the reader are exercised without a GPU;
the same round trip through Controller.run on the device is in
tests/test_gpu_api.py.
"""
import os

import numpy as np

import kat_setups as K
import pyclaw_b200 as pc

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _state(p, q, aux, t):
    x = pc.Dimension('x', -1.0, 1.0, p.mx)
    y = pc.Dimension('y', -1.0, 1.0, p.my)
    domain = pc.Domain([x, y])
    state = pc.State(domain, p.num_eqn, p.num_aux)
    state.q = np.asfortranarray(q)
    state.aux = np.asfortranarray(aux)
    state.t = t
    return pc.Solution(state, domain)


def test_oracle_frames_written_as_ascii_match_reference_files(orc, tmp_path):
    p, q, aux, run = K.acoustics_variable_setup()
    ref = orc.Run(p, q, aux, **run)
    frames = ref.run(0.6, num_output_times=20)
    out = str(tmp_path)
    _state(p, frames[0], aux, 0.0).write(0, out, 'ascii', write_aux=True)
    _state(p, frames[20], aux, ref.t).write(20, out, 'ascii')
    io = np.load(os.path.join(GOLD, "vc_acoustics_io.npz"))
    # header lines: identical text to the reference's files
    with open(os.path.join(out, "fort.t0020")) as f:
        assert f.read() == str(io["t_header"])
    with open(os.path.join(out, "fort.q0020")) as f:
        assert "\n".join(f.read().splitlines()[:8]) == str(io["q_header"])
    # read back as the reference's I/O test does, compare at its tolerance
    s0 = pc.Solution(0, path=out, file_format='ascii', read_aux=True)
    s20 = pc.Solution(20, path=out, file_format='ascii', read_aux=False)
    assert s20.state.t == 0.6 and s20.state.q.shape == (3, 200, 200)
    assert K.check_diff(io["q20"], s20.state.q, reltol=1e-4) is None
    assert K.check_diff(io["aux0"], s0.state.aux, reltol=1e-4) is None
    # the round trip keeps the %18.8e digits: relative error of one rounding
    got = s20.state.q
    big = np.abs(frames[20]) > 1e-300
    assert np.max(np.abs(got[big] - frames[20][big]) / np.abs(frames[20][big])) <= 5.1e-9
    assert s0.state.aux.shape == (2, 200, 200) and np.array_equal(s0.state.aux, aux)


def test_ascii_layout_rows_of_j_then_i(tmp_path):
    """Values run j-major, then i, one line per cell with num_eqn columns and a
    blank line after every row of the patch (io/ascii.py:85-99)."""
    p, q, aux, run = K.acoustics_variable_setup(mx=3, my=2)
    q = np.asfortranarray(np.arange(3 * 3 * 2, dtype=float).reshape(3, 3, 2, order='F') + 1.0)
    _state(p, q, aux, 0.25).write(7, str(tmp_path), 'ascii')
    lines = open(os.path.join(str(tmp_path), "fort.q0007")).read().splitlines()
    body = lines[9:]
    assert body[3] == "" and body[7] == ""
    vals = [[float(v) for v in ln.split()] for ln in body if ln]
    assert vals[0] == list(q[:, 0, 0]) and vals[1] == list(q[:, 1, 0]) and vals[3] == list(q[:, 0, 1])
    assert lines[2].split()[0] == "3" and lines[3].split()[0] == "2"
