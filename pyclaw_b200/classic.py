"""Classic Clawpack solvers: ClawSolver and ClawSolver2D (src/pyclaw/classic/solver.py).

ClawSolver2D keeps the reference's attributes and call contract
(step_hyperbolic advances the solution by dt and sets self.cfl), but the state
stays in GPU memory and the step is the fused sm_100a kernel of libclaw2.so.
evolve_to_time runs the whole step-size control loop on the device (one kernel
launch per step, no host round trip) unless a Python callback (before_step,
step_source, a custom boundary condition) has to run between steps; the
callbacks of pyclaw_b200.hooks (FixedStateBC, EulerRadialSource, AuxFromQ)
run on the device, and gauges are sampled on
the device after every accepted step and written out after each batch of
steps.
"""
import ctypes
import warnings

import numpy as np

from . import _abi
from . import _lib
from .limiters import tvd
from .solver import BC, Solver


class ClawSolver(Solver):
    def __init__(self, riemann_solver=None, claw_package=None):
        self.num_ghost = 2
        self.limiters = tvd.minmod
        self.order = 2
        self.source_split = 1
        self.fwave = False
        self.step_source = None
        self.before_step = None
        self.kernel_language = 'Fortran'
        self.verbosity = 0
        self.cfl_max = 1.0
        self.cfl_desired = 0.9
        self._mthlim = self.limiters
        self._method = None
        super(ClawSolver, self).__init__(riemann_solver, claw_package)

    # ClawSolver.step, classic/solver.py:100-151
    def step(self, solution):
        if self.before_step is not None:
            self.before_step(self, solution.states[0])
        if self.source_split == 2 and self.step_source is not None:
            self.step_source(self, solution.states[0], self.dt / 2.0)
        self.step_hyperbolic(solution)
        if self.cfl.get_cached_max() >= self.cfl_max:
            return False
        if self.step_source is not None:
            if self.source_split == 2:
                self.step_source(self, solution.states[0], self.dt / 2.0)
            if self.source_split == 1:
                self.step_source(self, solution.states[0], self.dt)
        return True

    def check_cfl_settings(self):
        pass

    def allocate_workspace(self, solution):
        pass

    def step_hyperbolic(self, solution):
        raise Exception("Dummy routine, please override!")

    def set_mthlim(self):
        self._mthlim = self.limiters
        if not isinstance(self.limiters, list):
            self._mthlim = [self._mthlim]
        if len(self._mthlim) == 1:
            self._mthlim = self._mthlim * self.num_waves
        if len(self._mthlim) != self.num_waves:
            raise Exception('Length of solver.limiters is not equal to 1 or to solver.num_waves')

    def set_method(self, state):
        self._method = np.empty(7, dtype=int, order='F')
        self._method[0] = self.dt_variable
        self._method[1] = self.order
        if self.num_dim == 1:
            self._method[2] = 0
        elif self.dimensional_split:
            self._method[2] = -1
        else:
            self._method[2] = self.transverse_waves
        self._method[3] = self.verbosity
        self._method[4] = 0
        self._method[5] = state.index_capa + 1
        self._method[6] = state.num_aux


class ClawSolver2D(ClawSolver):
    """2D classic (wave-propagation) solver on one B200."""

    no_trans = 0
    trans_inc = 1
    trans_cor = 2

    def __init__(self, riemann_solver=None, device=None):
        self.dimensional_split = True
        self.transverse_waves = self.trans_inc
        self.num_dim = 2
        self.aux1 = None
        self.aux2 = None
        self.aux3 = None
        self.work = None
        self.device = device
        self._dev = None
        self._problem = None
        super(ClawSolver2D, self).__init__(riemann_solver)

    def check_cfl_settings(self):
        if (not self.dimensional_split) and (self.transverse_waves == 0):
            cfl_recommended = 0.5
        else:
            cfl_recommended = 1.0
        if self.cfl_max > cfl_recommended:
            warnings.warn('cfl_max is set higher than the recommended value of %s' % cfl_recommended)
            warnings.warn(str(self.cfl_desired))

    # ---- setup ----------------------------------------------------------
    def make_problem(self, state):
        """Pack the solver's settings into the C ABI's claw2_problem
        (the information set_method/set_mthlim/set_cparam hand to step2)."""
        from . import riemann
        rp = self.rp
        if rp is None:
            raise Exception("solver.rp has not been set")
        if not isinstance(rp, riemann.RiemannSolver):
            name = getattr(rp, '__name__', str(rp)).split('.')[-1]
            if name not in riemann.SOLVERS:
                raise NotImplementedError("Riemann solver %s is not available on the GPU" % name)
            rp = riemann.SOLVERS[name]
        if self.num_waves is None:
            self.num_waves = rp.num_waves
        if state.num_eqn != rp.num_eqn or self.num_waves != rp.num_waves:
            raise Exception("num_eqn/num_waves do not match Riemann solver %s" % rp.name)
        if state.num_aux < rp.num_aux:
            raise Exception("Riemann solver %s needs %d aux fields" % (rp.name, rp.num_aux))
        self.set_mthlim()
        self.set_method(state)
        grid = state.grid
        mx, my = grid.num_cells
        dx, dy = grid.delta
        transverse = -1 if self.dimensional_split else int(self.transverse_waves)
        naux = state.num_aux
        aux_lo = [b if b is not None else BC.extrap for b in self.aux_bc_lower]
        aux_hi = [b if b is not None else BC.extrap for b in self.aux_bc_upper]
        if naux > 0 and (None in self.aux_bc_lower or None in self.aux_bc_upper):
            raise Exception("One or more of the aux boundary conditions has not been specified.")
        if None in self.bc_lower or None in self.bc_upper:
            raise Exception("One or more of the boundary conditions has not been specified.")
        return _abi.make_problem(
            rp=rp.rp_id, num_eqn=rp.num_eqn, num_waves=rp.num_waves, num_aux=naux, mx=mx, my=my,
            dx=dx, dy=dy, order=int(self.order), transverse=transverse,
            index_capa=int(state.index_capa), use_fwave=bool(self.fwave), mthlim=self._mthlim,
            bc_lower=self.bc_lower, bc_upper=self.bc_upper, aux_bc_lower=aux_lo, aux_bc_upper=aux_hi,
            params=rp.params(state.problem_data))

    def setup(self, solution):
        from .device import DeviceState
        state = solution.states[0]
        self.check_cfl_settings()
        self._problem = self.make_problem(state)
        rc = _lib.load().claw2_validate(ctypes.byref(self._problem))
        if rc == _abi.ERR_UNSUPPORTED:
            raise NotImplementedError("this problem configuration is not supported on the GPU: "
                                      "num_ghost must be 2 and periodic boundaries must be paired")
        _lib.check(rc, "claw2_validate")
        self._dev = DeviceState(self._problem, self.device)
        self._dev.attach(state)
        self._upload(state)
        self._is_set_up = True

    def _upload(self, state):
        dev = self._dev
        if dev.aux_dirty and state.num_aux > 0:
            dev.upload_aux(state._aux)
            if BC.custom in list(self.aux_bc_lower) + list(self.aux_bc_upper):
                g = self.num_ghost
                auxbc = np.zeros((state.num_aux, self._problem.mx + 2 * g, self._problem.my + 2 * g), order='F')
                auxbc[:, g:-g, g:-g] = state._aux
                self._fill_host_bcs(state, auxbc, self.aux_bc_lower, self.aux_bc_upper,
                                    self.user_aux_bc_lower,
                                    self.user_aux_bc_upper, negate=False)
                import torch
                v = dev.aux[:dev.L.aux_elems].view(state.num_aux, dev.L.rows, dev.L.ld)
                v[:, :, :auxbc.shape[1]].copy_(torch.from_numpy(np.ascontiguousarray(auxbc.transpose(0, 2, 1))))
        dev.aux_dirty = False
        dev.sync_from_host()

    def teardown(self):
        pass

    # ---- one step (used by the host-driven loop) -------------------------
    def _custom_bcs(self):
        return BC.custom in list(self.bc_lower) + list(self.bc_upper)

    def step_hyperbolic(self, solution):
        """classic/solver.py:498-545 on the device: fill ghost cells, step
        q[cur] -> q[1-cur], record the CFL number."""
        state = solution.states[0]
        if not self._is_set_up:
            self.setup(solution)
        dev = self._dev
        self._upload(state)
        if self._custom_bcs():
            qbc = dev.ghosted_ref()
            self._fill_host_bcs(state, qbc, self.bc_lower, self.bc_upper, self.user_bc_lower,
                                self.user_bc_upper, negate=True)
            dev.set_ghosted_ref(qbc)
        cfl, nxt = dev.step(self.dt)
        dev.cur = nxt
        dev.device_newer = True
        self.cfl.update_global_max(cfl)
        if np.isnan(cfl):
            raise FloatingPointError("the step produced a non-finite state")

    # ---- device-controlled loop ---------------------------------------------
    def _device_hooks(self):
        """The claw2_hooks that let the device run this solver's callbacks
        itself (hooks.EulerRadialSource, hooks.FixedStateBC), or None when
        some callback has to run on the host."""
        from .hooks import AuxFromQ, EulerRadialSource, FixedStateBC
        h = _abi.Hooks()
        if self.before_step is not None:
            if not isinstance(self.before_step, AuxFromQ):
                return None
            if list(self.aux_bc_lower) != list(self.bc_lower) or list(self.aux_bc_upper) != list(self.bc_upper):
                return None
            h.aux_from_q = self.before_step.aux_index + 1
            h.aux_q = self.before_step.q_index + 1
        if self.step_source is not None:
            if not isinstance(self.step_source, EulerRadialSource) or self.source_split != 1:
                return None
            h.source = self.step_source.kind
            h.source_aux = self.step_source.radius_aux
        for bcs, fns in ((self.bc_lower, self.user_bc_lower), (self.bc_upper, self.user_bc_upper)):
            if BC.custom in list(bcs) and not isinstance(fns, FixedStateBC):
                return None
        return h

    def _device_loop_ok(self, solution):
        return self._device_hooks() is not None

    def evolve_to_time(self, solution, tend=None):
        if not self._is_set_up:
            self.setup(solution)
        if not self._device_loop_ok(solution):
            return super(ClawSolver2D, self).evolve_to_time(solution, tend)
        state = solution.states[0]
        self._upload(state)
        take_one_step = tend is None
        lib = _lib.load()
        c = _abi.Control()
        rc = lib.claw2_control_init(ctypes.byref(c), float(solution.t), float(self.dt),
                                    float(tend if tend is not None else 0.0), float(self.cfl_max),
                                    float(self.cfl_desired), float(self.dt_max), int(bool(self.dt_variable)),
                                    int(take_one_step), int(self.max_steps), float(self.cfl.get_cached_max()))
        if rc != 0:
            if not self.dt_variable:
                raise Exception('dt does not divide (tend-tstart) and dt is fixed!')
            raise Exception('Variable time-stepping and desired CFL > maximum CFL')
        if not self.dt_variable:
            self.max_steps = int(c.max_steps)
        hooks = None
        if self.step_source is not None or self._custom_bcs() or self.before_step is not None:
            hooks = self._device_hooks()
            if self._custom_bcs():
                # fixed-state sides: set once in both state buffers; the
                # step never writes the ghost cells of custom sides
                dev = self._dev
                qbc = dev.ghosted_ref()
                self._fill_host_bcs(state, qbc, self.bc_lower, self.bc_upper, self.user_bc_lower,
                                    self.user_bc_upper, negate=True)
                dev.set_ghosted_ref(qbc, dev.cur)
                dev.set_ghosted_ref(qbc, 1 - dev.cur)
        gauges = [(int(g[0]), int(g[1])) for g in state.grid.gauges]
        on_gauges = None
        if gauges:
            # write_gauge_values after every accepted step (solver.py:654-656),
            # from samples the device recorded step by step
            def on_gauges(rows):
                for r in range(rows.shape[0]):
                    for i in range(len(gauges)):
                        self._write_gauge_sample(state, i, float(rows[r, i, 0]), rows[r, i, 1:])
        out = self._dev.evolve(c, hooks=hooks, gauges=gauges or None, on_gauges=on_gauges)
        solution.t = out.t
        self.dt = out.dt
        self.cfl.update_global_max(out.cfl)
        self.status['cflmax'] = out.status_cflmax
        self.status['dtmin'] = out.status_dtmin
        self.status['dtmax'] = out.status_dtmax
        self.status['numsteps'] = int(out.numsteps)
        if out.error == _abi.ERR_CFL:
            raise Exception('CFL too large, giving up!')
        if out.error == _abi.ERR_MAX_STEPS:
            raise Exception("Maximum number of timesteps have been taken")
        if out.error == _abi.ERR_NONFINITE:
            raise FloatingPointError("the step produced a non-finite state at t=%g" % out.t)
        if out.error:
            _lib.check(out.error, "device time-step loop")
        return self.status
