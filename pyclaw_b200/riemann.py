"""Riemann-solver descriptors for ``solver.rp``.

In the reference, ``solver.rp`` is an f2py module of the external
clawpack.riemann package whose Fortran rpn2/rpt2 are passed to step2 as
callbacks (src/pyclaw/classic/solver.py:518-519), with scalars copied into a
/cparam/ common block from ``state.problem_data`` (src/pyclaw/state.py:162-182)
and equation/wave counts looked up in ``riemann.static`` (src/pyclaw/solver.py:
206-211).  Device code cannot call Fortran callbacks, so here each solver is a
descriptor naming a compiled-in CUDA solver and the problem_data keys it needs.
"""
from . import _abi


class RiemannSolver(object):
    def __init__(self, name, rp_id, num_eqn, num_waves, num_aux, cparam):
        self.__name__ = 'clawpack.riemann.' + name
        self.name = name
        self.rp_id = rp_id
        self.num_eqn = num_eqn
        self.num_waves = num_waves
        self.num_aux = num_aux
        self.cparam = tuple(cparam)     # problem_data keys, in params[] order

    def params(self, problem_data):
        """problem_data -> params[] (missing keys raise like State.set_cparam)."""
        if not set(self.cparam) <= set(problem_data.keys()):
            raise Exception("Some required value(s) in the cparam common block in the Riemann "
                            "solver have not been set in problem_data.")
        return tuple(float(problem_data[k]) for k in self.cparam)

    def __repr__(self):
        return "<Riemann solver %s>" % self.name


rp2_acoustics = RiemannSolver('rp2_acoustics', _abi.RP_ACOUSTICS, 3, 2, 0, ('rho', 'bulk', 'cc', 'zz'))
rp2_vc_acoustics = RiemannSolver('rp2_vc_acoustics', _abi.RP_VC_ACOUSTICS, 3, 2, 2, ())
rp2_euler_4wave = RiemannSolver('rp2_euler_4wave', _abi.RP_EULER_4WAVE, 4, 4, 0, ('gamma', 'gamma1'))
rp2_euler_5wave = RiemannSolver('rp2_euler_5wave', _abi.RP_EULER_5WAVE, 5, 5, 0, ('gamma', 'gamma1'))
rp2_shallow_roe_with_efix = RiemannSolver('rp2_shallow_roe_with_efix', _abi.RP_SHALLOW_ROE, 3, 3, 0,
                                          ('grav',))

# f-wave solver (set solver.fwave = True, as apps/psystem_2d/psystem.py does);
# aux = (rho, K, linearity, eps), the application copies q[0] into aux[3]
# before each step
rp2_psystem = RiemannSolver('rp2_psystem', _abi.RP_PSYSTEM, 3, 2, 4, ())

SOLVERS = {s.name: s for s in (rp2_acoustics, rp2_vc_acoustics, rp2_euler_4wave, rp2_euler_5wave,
                               rp2_shallow_roe_with_efix, rp2_psystem)}


class static(object):
    """riemann.static: equation and wave counts by solver name."""
    num_eqn = {k: v.num_eqn for k, v in SOLVERS.items()}
    num_waves = {k: v.num_waves for k, v in SOLVERS.items()}
