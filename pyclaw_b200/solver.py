"""Solver base class: boundary-condition enum, attribute guard, status, and the
host-driven time-stepping loop (src/pyclaw/solver.py).

ClawSolver2D (classic.py) overrides evolve_to_time with a device-controlled loop
whenever no Python callback has to run between steps, and falls back to the
loop below (which still steps on the GPU, one kernel launch per step) when one
does.
"""
import logging

import numpy as np


class CFLError(Exception):
    def __init__(self, msg):
        super(CFLError, self).__init__(msg)


class BC(object):
    """Boundary condition names (solver.py:12-18)."""
    custom = 0
    extrap = 1
    periodic = 2
    wall = 3


def default_compute_gauge_values(q, aux):
    return q


class Solver(object):
    def __setattr__(self, key, value):
        if not hasattr(self, '_isinitialized'):
            self.__dict__['_isinitialized'] = False
        if self._isinitialized and not hasattr(self, key):
            raise TypeError("%s has no attribute %s" % (self.__class__, key))
        object.__setattr__(self, key, value)

    @property
    def all_bcs(self):
        return self.bc_lower, self.bc_upper

    @all_bcs.setter
    def all_bcs(self, all_bcs):
        for i in range(self.num_dim):
            self.bc_lower[i] = all_bcs
            self.bc_upper[i] = all_bcs

    def __init__(self, riemann_solver=None, claw_package=None):
        from .cfl import CFL
        self.logger = logging.getLogger('evolve')
        self.dt_initial = 0.1
        self.dt_max = 1e99
        self.max_steps = 10000
        self.dt_variable = True
        self.num_waves = None
        self.num_eqn = None
        self.qbc = None
        self.auxbc = None
        self.rp = None
        self.fmod = None
        self._is_set_up = False
        self.claw_package = None
        self.dt = self.dt_initial
        self.cfl = CFL(self.cfl_desired)
        self.status = {'cflmax': self.cfl.get_cached_max(), 'dtmin': self.dt,
                       'dtmax': self.dt, 'numsteps': 0}
        self.bc_lower = [None] * self.num_dim
        self.bc_upper = [None] * self.num_dim
        self.aux_bc_lower = [None] * self.num_dim
        self.aux_bc_upper = [None] * self.num_dim
        self.user_bc_lower = None
        self.user_bc_upper = None
        self.user_aux_bc_lower = None
        self.user_aux_bc_upper = None
        self.compute_gauge_values = default_compute_gauge_values
        if riemann_solver is not None:
            self.rp = riemann_solver
            from . import riemann
            name = riemann_solver.__name__.split('.')[-1]
            self.num_eqn = riemann.static.num_eqn[name]
            self.num_waves = riemann.static.num_waves[name]
        self._isinitialized = True

    def is_valid(self):
        valid = True
        if any(bc == BC.custom for bc in self.bc_lower) and self.user_bc_lower is None:
            self.logger.debug('Lower custom BC function has not been set.')
            valid = False
        if any(bc == BC.custom for bc in self.bc_upper) and self.user_bc_upper is None:
            self.logger.debug('Upper custom BC function has not been set.')
            valid = False
        return valid

    def setup(self, solution):
        pass

    def teardown(self):
        pass

    def __str__(self):
        out = "Solver Status:\n"
        for k, v in self.status.items():
            out = "\n".join((out, "%s = %s" % (k.rjust(25), v)))
        return out

    # ---- boundary conditions on a host qbc (reference semantics) ----------
    def _fill_host_bcs(self, state, qbc, lower, upper, user_lower, user_upper, negate):
        """apply_q_bcs / apply_aux_bcs (solver.py:299-365, 438-505) on a host
        ghosted array; x then y, lower then upper."""
        g = self.num_ghost
        for idim, dim in enumerate(state.grid.dimensions):
            for side in ('lower', 'upper'):
                bc = (lower if side == 'lower' else upper)[idim]
                if bc == BC.custom:
                    fn = user_lower if side == 'lower' else user_upper
                    fn(state, dim, state.t, qbc, g)
                    continue
                a = np.rollaxis(qbc, idim + 1, 1)
                if bc is None:
                    raise Exception("One or more of the boundary conditions has not been specified.")
                if side == 'lower':
                    if bc == BC.extrap:
                        for i in range(g):
                            a[:, i, ...] = a[:, g, ...]
                    elif bc == BC.periodic:
                        a[:, :g, ...] = a[:, -2 * g:-g, ...]
                    elif bc == BC.wall:
                        for i in range(g):
                            a[:, i, ...] = a[:, 2 * g - 1 - i, ...]
                            if negate:
                                a[idim + 1, i, ...] = -a[idim + 1, 2 * g - 1 - i, ...]
                    else:
                        raise NotImplementedError("Boundary condition %s not implemented" % bc)
                else:
                    if bc == BC.extrap:
                        for i in range(g):
                            a[:, -i - 1, ...] = a[:, -g - 1, ...]
                    elif bc == BC.periodic:
                        a[:, -g:, ...] = a[:, g:2 * g, ...]
                    elif bc == BC.wall:
                        for i in range(g):
                            a[:, -i - 1, ...] = a[:, -2 * g + i, ...]
                            if negate:
                                a[idim + 1, -i - 1, ...] = -a[idim + 1, -2 * g + i, ...]
                    else:
                        raise NotImplementedError("Boundary condition %s not implemented" % bc)

    # ---- host-driven loop (solver.py:582-699) -----------------------------
    def evolve_to_time(self, solution, tend=None):
        if not self._is_set_up:
            self.setup(solution)
        take_one_step = tend is None
        tstart = solution.t
        self.status['cflmax'] = self.cfl.get_cached_max()
        self.status['dtmin'] = self.dt
        self.status['dtmax'] = self.dt
        self.status['numsteps'] = 0
        if not self.dt_variable:
            if take_one_step:
                self.max_steps = 1
            else:
                self.max_steps = int((tend - tstart + 1e-10) / self.dt)
                if abs(self.max_steps * self.dt - (tend - tstart)) > 1e-5 * (tend - tstart):
                    raise Exception('dt does not divide (tend-tstart) and dt is fixed!')
        if self.dt_variable == 1 and self.cfl_desired > self.cfl_max:
            raise Exception('Variable time-stepping and desired CFL > maximum CFL')
        if not take_one_step and tend <= tstart:
            self.logger.info("Already at or beyond end time: no evolution required.")
            self.max_steps = 0
        for n in range(self.max_steps):
            state = solution.state
            if not take_one_step:
                if solution.t + self.dt > tend and tstart < tend:
                    self.dt = tend - solution.t
                if tend - solution.t - self.dt < 1.e-14 * solution.t:
                    self.dt = tend - solution.t
            if self.dt_variable:
                q_backup = state.q.copy('F')
                told = solution.t
            self.step(solution)
            cfl = self.cfl.get_cached_max()
            if cfl <= self.cfl_max:
                self.status['cflmax'] = max(cfl, self.status['cflmax'])
                if self.dt_variable:
                    solution.t += self.dt
                else:
                    solution.t = tstart + (n + 1) * self.dt
                self.logger.debug("Step %i  CFL = %f   dt = %f   t = %f" % (n, cfl, self.dt, solution.t))
                self.write_gauge_values(solution)
                self.status['numsteps'] += 1
            else:
                self.logger.debug("Rejecting time step, CFL number too large")
                if self.dt_variable:
                    state.q = q_backup
                    solution.t = told
                else:
                    self.status['cflmax'] = max(cfl, self.status['cflmax'])
                    raise Exception('CFL too large, giving up!')
            if self.dt_variable:
                if cfl > 0.0:
                    self.dt = min(self.dt_max, self.dt * self.cfl_desired / cfl)
                    self.status['dtmin'] = min(self.dt, self.status['dtmin'])
                    self.status['dtmax'] = max(self.dt, self.status['dtmax'])
                else:
                    self.dt = self.dt_max
            if take_one_step or solution.t >= tend:
                break
        if self.dt_variable and not take_one_step and solution.t < tend \
                and self.status['numsteps'] == self.max_steps:
            raise Exception("Maximum number of timesteps have been taken")
        return self.status

    def step(self, solution):
        raise NotImplementedError("No stepping routine has been defined!")

    # ---- gauges (solver.py:713-742) ----------------------------------------
    def write_gauge_values(self, solution):
        state = solution.state
        gauges = state.grid.gauges
        if not gauges:
            return
        dev = state._dev
        if dev is not None and dev.device_newer:
            qs = dev.cells_q(gauges)          # only the gauge cells leave the device
        else:
            qh = state.get_q_host()
            qs = np.stack([qh[:, g[0], g[1]] for g in gauges], axis=1)
        for i in range(len(gauges)):
            self._write_gauge_sample(state, i, solution.t, qs[:, i])

    def _write_gauge_sample(self, state, i, t, q):
        """One gauge's sample at time t: compute_gauge_values on q and the
        gauge cell's aux, kept in gauge_data and written to its file."""
        ix, iy = state.grid.gauges[i][0], state.grid.gauges[i][1]
        aux = state._aux[:, ix, iy] if state.num_aux > 0 else None
        p = self.compute_gauge_values(q, aux)
        if state.keep_gauges:
            gauge_data = state.gauge_data
            if len(gauge_data) == len(state.grid.gauges):
                gauge_data[i] = np.vstack((gauge_data[i], np.append(t, p)))
            else:
                gauge_data.append(np.append(t, p))
        try:
            state.grid.gauge_files[i].write(str(t) + ' ' + ' '.join(str(j) for j in p) + '\n')
        except Exception:
            raise Exception("Gauge files are not set up correctly. You should call the method "
                            "`setup_gauge_files` of the Grid class object before any call for "
                            "`write_gauge_values` from the Solver class.")
