"""ctypes binding and run driver for the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU arms import this
module.  The product package never does.

`Run` replays the reference driver loop in Python around the oracle's C step:
Controller.run (src/pyclaw/controller.py:202-316), Solver.evolve_to_time
(src/pyclaw/solver.py:582-699), ClawSolver.step (classic/solver.py:100-151)
and the Python boundary-condition fill Solver.apply_q_bcs (solver.py:299-434),
so that the reference's application scripts (custom boundary callbacks, source
terms) can be reproduced for the known-answer tests.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from pyclaw_b200 import _abi  # noqa: E402  (plain ctypes structs, no CUDA)

_LIBS = {}


def load(omp=False, timing=False):
    """Load (building if needed) the parity or the OpenMP oracle library, or
    with timing=True the host-native timing build (FMA allowed: for timing
    the CPU baseline only, never for parity; it has both the serial and the
    OpenMP entry points)."""
    key = "timing" if timing else ("omp" if omp else "serial")
    if key in _LIBS:
        return _LIBS[key]
    from oracle import build as _build  # noqa: WPS433
    if timing:
        path, flags, model = _build.build_timing()
        lib = ctypes.CDLL(path)
        lib.build_flags, lib.cpu_model = flags, model
        omp = True
    else:
        lib_path, omp_path = _build.build()
        lib = ctypes.CDLL(omp_path if omp else lib_path)
    P = ctypes.POINTER(_abi.Problem)
    dp = ctypes.POINTER(ctypes.c_double)
    C = ctypes.POINTER(_abi.Control)
    lib.orc_step2.argtypes = [P, dp, dp, dp, ctypes.c_double, dp]
    lib.orc_step2ds.argtypes = [P, dp, dp, dp, ctypes.c_double, ctypes.c_int, dp]
    lib.orc_fill_ghosts.argtypes = [P, dp]
    lib.orc_fill_aux_ghosts.argtypes = [P, dp]
    lib.orc_step_hyperbolic.argtypes = [P, dp, dp, dp, ctypes.c_double, dp]
    lib.orc_control_init.argtypes = [C, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_double]
    lib.orc_control_update.argtypes = [C, ctypes.c_double]
    lib.orc_evolve.argtypes = [P, dp, dp, C]
    for f in ("orc_step2", "orc_step2ds", "orc_fill_ghosts", "orc_fill_aux_ghosts",
              "orc_step_hyperbolic", "orc_control_init", "orc_control_update", "orc_evolve"):
        getattr(lib, f).restype = ctypes.c_int
    if omp:
        lib.orc_step_hyperbolic_omp.argtypes = [P, dp, dp, dp, ctypes.c_double, dp]
        lib.orc_step_hyperbolic_omp.restype = ctypes.c_int
        lib.orc_evolve_omp.argtypes = [P, dp, dp, C]
        lib.orc_evolve_omp.restype = ctypes.c_int
        lib.orc_num_threads.restype = ctypes.c_int
    _LIBS[key] = lib
    return lib


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed: %s" % (what, _abi.STATUS_TEXT.get(rc, rc)))


def qbc_shape(p, ncomp):
    g = p.num_ghost
    return (ncomp, p.mx + 2 * g, p.my + 2 * g)


def new_qbc(p, q=None, ncomp=None):
    """Ghosted Fortran-order array; interior set from q (ncomp, mx, my)."""
    ncomp = p.num_eqn if ncomp is None else ncomp
    a = np.zeros(qbc_shape(p, ncomp), order="F")
    if q is not None:
        g = p.num_ghost
        a[:, g:-g, g:-g] = q
    return a


def fill_ghosts(p, qbc, lib=None):
    lib = lib or load()
    _check(lib.orc_fill_ghosts(ctypes.byref(p), _dp(qbc)), "orc_fill_ghosts")


def fill_aux_ghosts(p, auxbc, lib=None):
    lib = lib or load()
    _check(lib.orc_fill_aux_ghosts(ctypes.byref(p), _dp(auxbc)), "orc_fill_aux_ghosts")


def step_hyperbolic(p, qbc, auxbc, dt, lib=None, omp=False):
    """qbc (ghost-filled) is advanced in place; returns the CFL number."""
    lib = lib or load(omp)
    work = np.empty_like(qbc, order="F")
    cfl = ctypes.c_double(0.0)
    fn = lib.orc_step_hyperbolic_omp if omp else lib.orc_step_hyperbolic
    _check(fn(ctypes.byref(p), _dp(qbc), _dp(work), _dp(auxbc), float(dt), ctypes.byref(cfl)),
           "orc_step_hyperbolic")
    return cfl.value


def step2(p, qold, qnew, aux, dt, lib=None):
    lib = lib or load()
    cfl = ctypes.c_double(0.0)
    _check(lib.orc_step2(ctypes.byref(p), _dp(qold), _dp(qnew), _dp(aux), float(dt),
                         ctypes.byref(cfl)), "orc_step2")
    return cfl.value


def step2ds(p, qold, qnew, aux, dt, ids, lib=None):
    lib = lib or load()
    cfl = ctypes.c_double(0.0)
    _check(lib.orc_step2ds(ctypes.byref(p), _dp(qold), _dp(qnew), _dp(aux), float(dt), int(ids),
                           ctypes.byref(cfl)), "orc_step2ds")
    return cfl.value


def control_init(t, dt, tend, cfl_max, cfl_desired, dt_max=1e99, dt_variable=True,
                 take_one_step=False, max_steps=10000, prev_cfl=None, lib=None):
    lib = lib or load()
    c = _abi.Control()
    prev = cfl_desired if prev_cfl is None else prev_cfl
    _check(lib.orc_control_init(ctypes.byref(c), t, dt, tend, cfl_max, cfl_desired, dt_max,
                                int(dt_variable), int(take_one_step), int(max_steps), prev),
           "orc_control_init")
    return c


def evolve(p, qbc, auxbc, ctrl, omp=False, lib=None):
    """C replay of evolve_to_time (non-custom BCs, no source term)."""
    lib = lib or load(omp)
    fn = lib.orc_evolve_omp if omp else lib.orc_evolve
    rc = fn(ctypes.byref(p), _dp(qbc), _dp(auxbc), ctypes.byref(ctrl))
    return rc


class Run:
    """Python replay of Controller.run + evolve_to_time around the oracle step.

    bc_callbacks: {(idim, 'lower'|'upper'): f(qbc, t)} for CUSTOM sides; f
    receives the unrolled ghosted array, like user_bc_lower/upper do
    (solver.py:344-357).  step_source(q_interior_view, dt) mirrors
    solver.step_source (classic/solver.py:142-149; Godunov splitting).
    """

    def __init__(self, p, q, aux=None, *, cfl_max=1.0, cfl_desired=0.9, dt_initial=0.1,
                 dt_max=1e99, dt_variable=True, max_steps=10000, bc_callbacks=None,
                 step_source=None, source_split=1, lib=None, omp=False, before_step=None,
                 on_accept=None):
        self.p = p
        self.omp = omp
        self.lib = lib or load(omp)
        g = p.num_ghost
        self.qbc = new_qbc(p, q)
        self.q = self.qbc[:, g:-g, g:-g]
        self.auxbc = None
        if p.num_aux > 0:
            self.auxbc = new_qbc(p, aux, p.num_aux)
            fill_aux_ghosts(p, self.auxbc, self.lib)
        self.cfl_max = cfl_max
        self.cfl_desired = cfl_desired
        self.dt = dt_initial
        self.dt_max = dt_max
        self.dt_variable = dt_variable
        self.max_steps = max_steps
        self.bc_callbacks = bc_callbacks or {}
        self.step_source = step_source
        self.source_split = source_split
        self.before_step = before_step      # f(run): may change the interior of run.auxbc
        self.on_accept = on_accept          # f(run) after every accepted step (gauges)
        self.t = 0.0
        self.cfl = cfl_desired           # CFL(cfl_desired), solver.py:179
        self.status = {}
        self.steps_taken = 0
        self.dts = []

    # Solver.apply_q_bcs (solver.py:299-365): x then y, lower then upper
    def apply_q_bcs(self):
        p, g = self.p, self.p.num_ghost
        qbc = self.qbc
        qbc[:, g:-g, g:-g] = self.q
        for idim in range(2):
            for side in ("lower", "upper"):
                bc = (p.bc_lower if side == "lower" else p.bc_upper)[idim]
                if bc == _abi.BC_CUSTOM:
                    self.bc_callbacks[(idim, side)](qbc, self.t)
                    continue
                a = np.moveaxis(qbc, idim + 1, 1)
                if side == "lower":
                    if bc == _abi.BC_EXTRAP:
                        for i in range(g):
                            a[:, i, ...] = a[:, g, ...]
                    elif bc == _abi.BC_PERIODIC:
                        a[:, :g, ...] = a[:, -2 * g:-g, ...]
                    elif bc == _abi.BC_WALL:
                        for i in range(g):
                            a[:, i, ...] = a[:, 2 * g - 1 - i, ...]
                            a[idim + 1, i, ...] = -a[idim + 1, 2 * g - 1 - i, ...]
                else:
                    if bc == _abi.BC_EXTRAP:
                        for i in range(g):
                            a[:, -i - 1, ...] = a[:, -g - 1, ...]
                    elif bc == _abi.BC_PERIODIC:
                        a[:, -g:, ...] = a[:, g:2 * g, ...]
                    elif bc == _abi.BC_WALL:
                        for i in range(g):
                            a[:, -i - 1, ...] = a[:, -2 * g + i, ...]
                            a[idim + 1, -i - 1, ...] = -a[idim + 1, -2 * g + i, ...]

    def step(self):
        """ClawSolver.step (classic/solver.py:100-151); returns True on success."""
        if self.before_step is not None:            # classic/solver.py:128-129
            self.before_step(self)
            fill_aux_ghosts(self.p, self.auxbc, self.lib)    # apply_aux_bcs in step_hyperbolic
        self.apply_q_bcs()
        self.cfl = step_hyperbolic(self.p, self.qbc, self.auxbc, self.dt, lib=self.lib, omp=self.omp)
        g = self.p.num_ghost
        self.q = self.qbc[:, g:-g, g:-g]
        if self.cfl >= self.cfl_max:
            return False
        if self.step_source is not None:
            if self.source_split == 2:
                self.step_source(self.q, self.dt / 2.0)
            elif self.source_split == 1:
                self.step_source(self.q, self.dt)
        return True

    def evolve_to_time(self, tend=None):
        """Solver.evolve_to_time (solver.py:582-699), literally."""
        take_one_step = tend is None
        tstart = self.t
        self.status = {"cflmax": self.cfl, "dtmin": self.dt, "dtmax": self.dt, "numsteps": 0}
        max_steps = self.max_steps
        if not self.dt_variable:
            if take_one_step:
                max_steps = 1
            else:
                max_steps = int((tend - tstart + 1e-10) / self.dt)
                if abs(max_steps * self.dt - (tend - tstart)) > 1e-5 * (tend - tstart):
                    raise Exception('dt does not divide (tend-tstart) and dt is fixed!')
        if self.dt_variable == 1 and self.cfl_desired > self.cfl_max:
            raise Exception('Variable time-stepping and desired CFL > maximum CFL')
        if not take_one_step and tend <= tstart:
            max_steps = 0
        for n in range(max_steps):
            if not take_one_step:
                if self.t + self.dt > tend and tstart < tend:
                    self.dt = tend - self.t
                if tend - self.t - self.dt < 1.e-14 * self.t:
                    self.dt = tend - self.t
            if self.dt_variable:
                q_backup = self.q.copy("F")
                told = self.t
            self.step()
            self.dts.append(self.dt)
            cfl = self.cfl
            if cfl <= self.cfl_max:
                self.status["cflmax"] = max(cfl, self.status["cflmax"])
                if self.dt_variable:
                    self.t += self.dt
                else:
                    self.t = tstart + (n + 1) * self.dt
                self.status["numsteps"] += 1
                self.steps_taken += 1
                if self.on_accept is not None:      # write_gauge_values, solver.py:654-656
                    self.on_accept(self)
            else:
                if self.dt_variable:
                    self.q = q_backup
                    self.t = told
                else:
                    self.status["cflmax"] = max(cfl, self.status["cflmax"])
                    raise Exception('CFL too large, giving up!')
            if self.dt_variable:
                if cfl > 0.0:
                    self.dt = min(self.dt_max, self.dt * self.cfl_desired / cfl)
                    self.status["dtmin"] = min(self.dt, self.status["dtmin"])
                    self.status["dtmax"] = max(self.dt, self.status["dtmax"])
                else:
                    self.dt = self.dt_max
            if take_one_step or self.t >= tend:
                break
        if self.dt_variable and not take_one_step and self.t < tend \
                and self.status["numsteps"] == max_steps:
            raise Exception("Maximum number of timesteps have been taken")
        return self.status

    def run(self, tfinal, num_output_times=10, keep_copy=True):
        """Controller.run with output_style 1 (controller.py:240-289)."""
        frames = [self.q.copy("F")] if keep_copy else []
        times = np.linspace(self.t, tfinal, num_output_times + 1)
        for t in times[1:]:
            self.evolve_to_time(t)
            if keep_copy:
                frames.append(self.q.copy("F"))
        return frames
