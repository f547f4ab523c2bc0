"""ctypes mirrors of the plain-data structs in include/claw2.h.

The field order and types must match the C declarations exactly; the
module-level asserts below check the sizes the C side reports at load time
(see pyclaw_b200._lib).
"""
import ctypes

ABI_VERSION = 1
MAX_EQN = 8
MAX_WAVES = 8
MAX_PARAMS = 8
NUM_GHOST = 2

# status codes (enum claw2_status)
OK = 0
ERR_INVALID = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_CFL = 4
ERR_MAX_STEPS = 5
ERR_NONFINITE = 6
ERR_TIMEOUT = 7
ERR_NOMEM = 8
ERR_SIZE = 9

# Riemann solver ids (enum claw2_rp)
RP_ACOUSTICS = 1
RP_VC_ACOUSTICS = 2
RP_EULER_4WAVE = 3
RP_EULER_5WAVE = 4
RP_SHALLOW_ROE = 5
RP_PSYSTEM = 6

# boundary conditions (enum claw2_bc == pyclaw.BC)
BC_CUSTOM = 0
BC_EXTRAP = 1
BC_PERIODIC = 2
BC_WALL = 3


class Problem(ctypes.Structure):
    """struct claw2_problem."""
    _fields_ = [
        ("rp", ctypes.c_int32),
        ("num_eqn", ctypes.c_int32),
        ("num_waves", ctypes.c_int32),
        ("num_aux", ctypes.c_int32),
        ("mx", ctypes.c_int32),
        ("my", ctypes.c_int32),
        ("num_ghost", ctypes.c_int32),
        ("order", ctypes.c_int32),
        ("transverse", ctypes.c_int32),
        ("index_capa", ctypes.c_int32),
        ("use_fwave", ctypes.c_int32),
        ("mthlim", ctypes.c_int32 * MAX_WAVES),
        ("bc_lower", ctypes.c_int32 * 2),
        ("bc_upper", ctypes.c_int32 * 2),
        ("aux_bc_lower", ctypes.c_int32 * 2),
        ("aux_bc_upper", ctypes.c_int32 * 2),
        ("dx", ctypes.c_double),
        ("dy", ctypes.c_double),
        ("params", ctypes.c_double * MAX_PARAMS),
    ]


# source terms of claw2_hooks (enum claw2_source)
SRC_NONE = 0
SRC_EULER_RADIAL = 1


class Hooks(ctypes.Structure):
    """struct claw2_hooks."""
    _fields_ = [
        ("source", ctypes.c_int32),
        ("source_aux", ctypes.c_int32),
        ("aux_from_q", ctypes.c_int32),
        ("aux_q", ctypes.c_int32),
    ]


class Gauges(ctypes.Structure):
    """struct claw2_gauges (device pointers)."""
    _fields_ = [
        ("ngauges", ctypes.c_int32),
        ("capacity", ctypes.c_int32),
        ("cells", ctypes.c_void_p),
        ("record", ctypes.c_void_p),
        ("state", ctypes.c_void_p),
    ]


class Layout(ctypes.Structure):
    """struct claw2_layout."""
    _fields_ = [
        ("ld", ctypes.c_int64),
        ("rows", ctypes.c_int64),
        ("plane", ctypes.c_int64),
        ("q_elems", ctypes.c_int64),
        ("aux_elems", ctypes.c_int64),
    ]


class Control(ctypes.Structure):
    """struct claw2_control (device-resident time-step controller)."""
    _fields_ = [
        ("t", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("tstart", ctypes.c_double),
        ("tend", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("cfl_max", ctypes.c_double),
        ("cfl_desired", ctypes.c_double),
        ("dt_max", ctypes.c_double),
        ("status_cflmax", ctypes.c_double),
        ("status_dtmin", ctypes.c_double),
        ("status_dtmax", ctypes.c_double),
        ("numsteps", ctypes.c_int64),
        ("iter", ctypes.c_int64),
        ("max_steps", ctypes.c_int64),
        ("rejected", ctypes.c_int64),
        ("cur", ctypes.c_int32),
        ("done", ctypes.c_int32),
        ("error", ctypes.c_int32),
        ("dt_variable", ctypes.c_int32),
        ("take_one_step", ctypes.c_int32),
        ("reserved_", ctypes.c_uint32),
        ("pad_", ctypes.c_int32 * 2),
    ]


assert ctypes.sizeof(Control) == 11 * 8 + 4 * 8 + 8 * 4, ctypes.sizeof(Control)

STATUS_TEXT = {
    OK: "ok",
    ERR_INVALID: "invalid problem description or argument",
    ERR_UNSUPPORTED: "feature not supported by this build",
    ERR_CUDA: "CUDA runtime error",
    ERR_CFL: "CFL too large, giving up!",
    ERR_MAX_STEPS: "Maximum number of timesteps have been taken",
    ERR_NONFINITE: "non-finite or non-physical state produced",
    ERR_TIMEOUT: "bounded device wait gave up",
    ERR_NOMEM: "out of memory",
    ERR_SIZE: "size beyond the documented maximum",
}


def make_problem(*, rp, num_eqn, num_waves, num_aux, mx, my, dx, dy, order=2,
                 transverse=1, index_capa=-1, use_fwave=False, mthlim=(1,),
                 bc_lower=(BC_EXTRAP, BC_EXTRAP), bc_upper=(BC_EXTRAP, BC_EXTRAP),
                 aux_bc_lower=(BC_EXTRAP, BC_EXTRAP), aux_bc_upper=(BC_EXTRAP, BC_EXTRAP),
                 params=()):
    """Build a Problem from keyword settings (limiter list broadcast as
    ClawSolver.set_mthlim does, src/pyclaw/classic/solver.py:167-176)."""
    p = Problem()
    p.rp = rp
    p.num_eqn = num_eqn
    p.num_waves = num_waves
    p.num_aux = num_aux
    p.mx = mx
    p.my = my
    p.num_ghost = NUM_GHOST
    p.order = order
    p.transverse = transverse
    p.index_capa = index_capa
    p.use_fwave = int(bool(use_fwave))
    lim = list(mthlim)
    if len(lim) == 1:
        lim = lim * num_waves
    if len(lim) != num_waves:
        raise Exception('Length of solver.limiters is not equal to 1 or to solver.num_waves')
    for k, v in enumerate(lim):
        p.mthlim[k] = int(v)
    for k in range(2):
        p.bc_lower[k] = int(bc_lower[k])
        p.bc_upper[k] = int(bc_upper[k])
        p.aux_bc_lower[k] = int(aux_bc_lower[k])
        p.aux_bc_upper[k] = int(aux_bc_upper[k])
    p.dx = float(dx)
    p.dy = float(dy)
    for k, v in enumerate(params):
        p.params[k] = float(v)
    return p
