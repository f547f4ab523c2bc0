"""Device-side forms of application callbacks.

The reference's applications pass Python functions for boundary conditions
(solver.user_bc_lower/upper) and source terms (solver.step_source).  Those
run on the host between steps, which forces ClawSolver2D onto its
host-driven loop (a device-host round trip per step).  The two classes here
are ordinary callbacks with the reference's signatures, so they work the same
on the host path, and ClawSolver2D recognises them and keeps the whole
evolve_to_time loop on the device:

* ``FixedStateBC(values, side)``: ghost cells of one side held at a constant
  state, like the shock-bubble app's inflow condition
  (apps/euler_2d/shockbubble.py:68-87).
* ``EulerRadialSource(radius_aux=0)``: the geometric source of the Euler
  equations with radial symmetry, two-stage Runge-Kutta
  (apps/euler_2d/shockbubble.py:89-124), fused into the step kernel.  Used
  with Godunov splitting (solver.source_split = 1).
* ``AuxFromQ(aux_index=3, q_index=0)``: a before_step callback that copies a
  state component into an aux component the Riemann solver reads, like the
  p-system app's b4step (apps/psystem_2d/psystem.py:86-90, aux[3] = q[0] for
  its transverse solver); on the device a copy kernel runs before each step.
"""
import numpy as np

from . import _abi


class FixedStateBC(object):
    """Custom boundary condition: every ghost layer of the side `side`
    ("lower" or "upper") of the dimension it is attached to holds `values`
    (one number per equation)."""

    def __init__(self, values, side="lower"):
        if side not in ("lower", "upper"):
            raise ValueError("side must be 'lower' or 'upper'")
        self.values = np.asarray(values, dtype=np.float64)
        self.side = side

    def __call__(self, state, dim, t, qbc, num_ghost):
        names = [d.name for d in state.grid.dimensions]
        axis = names.index(dim.name) + 1
        a = np.rollaxis(qbc, axis, 1)
        if self.values.shape[0] != a.shape[0]:
            raise ValueError("FixedStateBC has %d values for %d equations" % (self.values.shape[0], a.shape[0]))
        for i in range(num_ghost):
            k = i if self.side == "lower" else -1 - i
            a[:, k, ...] = self.values.reshape((-1,) + (1,) * (a.ndim - 2))


class EulerRadialSource(object):
    """step_source(solver, state, dt) for the Euler equations with radial
    symmetry, the radial coordinate in aux[radius_aux]; on the device it is
    applied inside the step kernel."""

    kind = _abi.SRC_EULER_RADIAL

    def __init__(self, radius_aux=0):
        self.radius_aux = int(radius_aux)

    def __call__(self, solver, state, dt):
        gamma1 = state.problem_data['gamma1']
        q = state.q
        rad = state.aux[self.radius_aux, :, :]
        dt2 = dt / 2.
        ndim = 2
        rho = q[0, :, :]
        u = q[1, :, :] / rho
        v = q[2, :, :] / rho
        press = gamma1 * (q[3, :, :] - 0.5 * rho * (u ** 2 + v ** 2))
        qstar = np.empty(q.shape)
        qstar[0, :, :] = q[0, :, :] - dt2 * (ndim - 1) / rad * q[2, :, :]
        qstar[1, :, :] = q[1, :, :] - dt2 * (ndim - 1) / rad * rho * u * v
        qstar[2, :, :] = q[2, :, :] - dt2 * (ndim - 1) / rad * rho * v * v
        qstar[3, :, :] = q[3, :, :] - dt2 * (ndim - 1) / rad * v * (q[3, :, :] + press)
        rho = qstar[0, :, :]
        u = qstar[1, :, :] / rho
        v = qstar[2, :, :] / rho
        press = gamma1 * (qstar[3, :, :] - 0.5 * rho * (u ** 2 + v ** 2))
        q[0, :, :] = q[0, :, :] - dt * (ndim - 1) / rad * qstar[2, :, :]
        q[1, :, :] = q[1, :, :] - dt * (ndim - 1) / rad * rho * u * v
        q[2, :, :] = q[2, :, :] - dt * (ndim - 1) / rad * rho * v * v
        q[3, :, :] = q[3, :, :] - dt * (ndim - 1) / rad * v * (qstar[3, :, :] + press)


class AuxFromQ(object):
    """before_step(solver, state): state.aux[aux_index] = state.q[q_index].
    On the device loop the copy runs before every step, ghost cells included,
    which needs the aux boundary conditions of that component to equal those
    of q (ClawSolver2D falls back to the host loop otherwise)."""

    def __init__(self, aux_index=3, q_index=0):
        self.aux_index = int(aux_index)
        self.q_index = int(q_index)

    def __call__(self, solver, state):
        state.aux[self.aux_index, :, :] = state.q[self.q_index, :, :]
