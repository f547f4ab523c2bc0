"""Clawpack ascii frame files fort.tXXXX / fort.qXXXX / fort.aXXXX
(src/pyclaw/io/ascii.py:14-395): same header lines, same %18.8e values, j-major
then i then m, with a blank line after every row of the patch."""
import os

import numpy as np


def _header(f, patch):
    f.write("%5i                  patch_number\n" % patch.patch_index)
    f.write("%5i                  AMR_level\n" % patch.level)
    for dim in patch.dimensions:
        f.write("%5i                  m%s\n" % (dim.num_cells, dim.name))
    for dim in patch.dimensions:
        f.write("%18.8e     %slow\n" % (dim.lower, dim.name))
    for dim in patch.dimensions:
        f.write("%18.8e     d%s\n" % (dim.delta, dim.name))
    f.write("\n")


def _body(f, a):
    """a: (nvar, mx, my); rows of j, each a block of i lines of nvar values."""
    nvar, mx, my = a.shape
    fmt = "%18.8e" * nvar
    for j in range(my):
        rows = a[:, :, j].T
        f.write("\n".join(fmt % tuple(r) for r in rows))
        f.write("\n\n")


def write(solution, frame, path, file_prefix='fort', write_aux=False, options={}, write_p=False):
    with open(os.path.join(path, '%s.t%s' % (file_prefix, str(frame).zfill(4))), 'w') as f:
        f.write("%18.8e     time\n" % solution.t)
        f.write("%5i                  num_eqn\n" % solution.num_eqn)
        f.write("%5i                  nstates\n" % len(solution.states))
        f.write("%5i                  num_aux\n" % solution.num_aux)
        f.write("%5i                  num_dim\n" % solution.domain.num_dim)
    with open(os.path.join(path, 'fort.q%s' % str(frame).zfill(4)), 'w') as f:
        for state in solution.states:
            _header(f, state.patch)
            q = state.p if write_p else state.get_q_host()
            _body(f, np.asarray(q))
    if solution.num_aux > 0 and write_aux:
        with open(os.path.join(path, 'fort.a%s' % str(frame).zfill(4)), 'w') as f:
            for state in solution.states:
                _header(f, state.patch)
                _body(f, np.asarray(state._aux))


def _read_patch(lines, nvar):
    mx = int(lines[2].split()[0])
    my = int(lines[3].split()[0])
    xlow = float(lines[4].split()[0]); ylow = float(lines[5].split()[0])
    dx = float(lines[6].split()[0]); dy = float(lines[7].split()[0])
    vals = np.array([float(v) for ln in lines[8:] for v in ln.split()])
    a = vals[:mx * my * nvar].reshape(my, mx, nvar).transpose(2, 1, 0)
    return np.asfortranarray(a), (mx, my, xlow, ylow, dx, dy)


def read(solution, frame, path='./', file_prefix='fort', read_aux=True, options={}):
    from ..geometry import Dimension, Domain
    from ..state import State
    with open(os.path.join(path, '%s.t%s' % (file_prefix, str(frame).zfill(4)))) as f:
        t = float(f.readline().split()[0])
        num_eqn = int(f.readline().split()[0])
        f.readline()
        num_aux = int(f.readline().split()[0])
    with open(os.path.join(path, 'fort.q%s' % str(frame).zfill(4))) as f:
        lines = f.read().splitlines()
    q, (mx, my, xlow, ylow, dx, dy) = _read_patch(lines, num_eqn)
    x = Dimension('x', xlow, xlow + mx * dx, mx)
    y = Dimension('y', ylow, ylow + my * dy, my)
    domain = Domain([x, y])
    aux = None
    apath = os.path.join(path, 'fort.a%s' % str(frame).zfill(4))
    if read_aux and num_aux > 0 and os.path.exists(apath):
        with open(apath) as f:
            aux, _ = _read_patch(f.read().splitlines(), num_aux)
    state = State(domain, num_eqn, num_aux if aux is not None else 0)
    state.q = q
    if aux is not None:
        state.aux = aux
    state.t = t
    solution.states = [state]
    solution.domain = domain
