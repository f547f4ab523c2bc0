"""pyclaw_b200 -- PyClaw's 2D classic wave-propagation step on NVIDIA B200 (sm_100a).

The public names mirror ``clawpack.pyclaw`` (src/pyclaw/__init__.py):

    from pyclaw_b200 import pyclaw-style classes
    solver = ClawSolver2D(); solver.rp = riemann.rp2_euler_4wave; ...
    claw = Controller(); claw.solution = Solution(state, domain); claw.run()

The step itself runs as hand-written CUDA kernels from libclaw2.so (built by
``python -m pyclaw_b200.build``); there is no CPU fallback.
"""
from . import hooks, limiters, riemann  # noqa: F401
from .cfl import CFL  # noqa: F401
from .classic import ClawSolver, ClawSolver2D  # noqa: F401
from .controller import Controller  # noqa: F401
from .geometry import Dimension, Domain, Grid, Patch  # noqa: F401
from .solution import Solution  # noqa: F401
from .solver import BC, CFLError, Solver  # noqa: F401
from .state import State  # noqa: F401

__version__ = "0.1.0"
