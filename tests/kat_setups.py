"""The reference's 2D application setups, restated in Python 3 for the
known-answer tests (initial data, boundary callbacks, source terms and solver
settings).  Each builder cites the reference script it follows.  Grids follow
pyclaw.Dimension: delta = (upper-lower)/num_cells, centers[i] = lower +
(i+0.5)*delta (src/pyclaw/geometry.py:425-446).
"""
import numpy as np

from pyclaw_b200 import _abi


def centers(lower, upper, n):
    delta = (upper - lower) / float(n)
    c = np.empty(n)
    for i in range(n):
        c[i] = lower + (i + 0.5) * delta
    return c, delta


# --------------------------------------------------------------------------
# apps/euler_2d/shockbubble.py (classic solver branch, :157-235)
# --------------------------------------------------------------------------
GAMMA = 1.4
GAMMA1 = GAMMA - 1.


def _shock_state(pinf=5.):
    rinf = (GAMMA1 + pinf * (GAMMA + 1.)) / ((GAMMA + 1.) + GAMMA1 * pinf)
    vinf = 1. / np.sqrt(GAMMA) * (pinf - 1.) / np.sqrt(0.5 * ((GAMMA + 1.) / GAMMA) * pinf + 0.5 * GAMMA1 / GAMMA)
    einf = 0.5 * rinf * vinf ** 2 + pinf / GAMMA1
    return rinf, vinf, einf


def shockbubble_setup(mx=160, my=40):
    """Returns (problem, q0, aux0, run_kwargs, bc_callbacks, step_source)."""
    from scipy import integrate
    x, dx = centers(0.0, 2.0, mx)
    y, dy = centers(0.0, 0.5, my)
    x0, y0, r0 = 0.5, 0., 0.2
    xshock = 0.2
    rhoin, pinf = 0.1, 5.
    rhoout, pout, pin = 1., 1., 1.
    rinf, vinf, einf = _shock_state(pinf)

    def ycirc(xx, ymin, ymax):                       # shockbubble.py:11-15
        if ((xx - x0) ** 2) < (r0 ** 2):
            return max(min(y0 + np.sqrt(r0 ** 2 - (xx - x0) ** 2), ymax) - ymin, 0.)
        return 0

    q = np.empty((5, mx, my), order="F")             # qinit, :17-57
    Y, X = np.meshgrid(y, x)
    r = np.sqrt((X - x0) ** 2 + (Y - y0) ** 2)
    q[0, :, :] = rinf * (X < xshock) + rhoin * (r <= r0) + rhoout * (r > r0) * (X >= xshock)
    q[1, :, :] = rinf * vinf * (X < xshock)
    q[2, :, :] = 0.
    q[3, :, :] = einf * (X < xshock) + (pin * (r <= r0) + pout * (r > r0) * (X >= xshock)) / GAMMA1
    q[4, :, :] = 1. * (r <= r0)
    d2 = np.linalg.norm([dx, dy]) / 2.
    dx2, dy2 = dx / 2., dy / 2.
    for i in range(mx):
        for j in range(my):
            ydown = y[j] - dy2
            yup = y[j] + dy2
            if abs(r[i, j] - r0) < d2:
                infrac, abserr = integrate.quad(ycirc, x[i] - dx2, x[i] + dx2, args=(ydown, yup),
                                                epsabs=1.e-8, epsrel=1.e-5)
                infrac = infrac / (dx * dy)
                q[0, i, j] = rhoin * infrac + rhoout * (1. - infrac)
                q[3, i, j] = (pin * infrac + pout * (1. - infrac)) / GAMMA1
                q[4, i, j] = 1. * infrac
    aux = np.empty((1, mx, my), order="F")           # auxinit, :59-66
    for j, yc in enumerate(y):
        aux[0, :, j] = yc

    def shockbc(qbc, t):                             # :68-87 (lower x, custom)
        for i in range(2):
            qbc[0, i, ...] = rinf
            qbc[1, i, ...] = rinf * vinf
            qbc[2, i, ...] = 0.
            qbc[3, i, ...] = einf
            qbc[4, i, ...] = 0.

    def step_Euler_radial(qv, dt):                   # :89-124
        dt2 = dt / 2.
        ndim = 2
        rad = aux[0, :, :]
        rho = qv[0, :, :]
        u = qv[1, :, :] / rho
        v = qv[2, :, :] / rho
        press = GAMMA1 * (qv[3, :, :] - 0.5 * rho * (u ** 2 + v ** 2))
        qstar = np.empty(qv.shape)
        qstar[0, :, :] = qv[0, :, :] - dt2 * (ndim - 1) / rad * qv[2, :, :]
        qstar[1, :, :] = qv[1, :, :] - dt2 * (ndim - 1) / rad * rho * u * v
        qstar[2, :, :] = qv[2, :, :] - dt2 * (ndim - 1) / rad * rho * v * v
        qstar[3, :, :] = qv[3, :, :] - dt2 * (ndim - 1) / rad * v * (qv[3, :, :] + press)
        rho = qstar[0, :, :]
        u = qstar[1, :, :] / rho
        v = qstar[2, :, :] / rho
        press = GAMMA1 * (qstar[3, :, :] - 0.5 * rho * (u ** 2 + v ** 2))
        qv[0, :, :] = qv[0, :, :] - dt * (ndim - 1) / rad * qstar[2, :, :]
        qv[1, :, :] = qv[1, :, :] - dt * (ndim - 1) / rad * rho * u * v
        qv[2, :, :] = qv[2, :, :] - dt * (ndim - 1) / rad * rho * v * v
        qv[3, :, :] = qv[3, :, :] - dt * (ndim - 1) / rad * v * (qstar[3, :, :] + press)

    p = _abi.make_problem(
        rp=_abi.RP_EULER_5WAVE, num_eqn=5, num_waves=5, num_aux=1, mx=mx, my=my, dx=dx, dy=dy,
        order=2, transverse=-1, mthlim=[4, 4, 4, 4, 2],
        bc_lower=(_abi.BC_CUSTOM, _abi.BC_WALL), bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP),
        aux_bc_lower=(_abi.BC_EXTRAP, _abi.BC_EXTRAP), aux_bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP),
        params=(GAMMA, GAMMA1))
    run = dict(cfl_max=0.5, cfl_desired=0.45, dt_initial=0.005, source_split=1)
    return p, q, aux, run, {(0, "lower"): shockbc}, step_Euler_radial


# --------------------------------------------------------------------------
# apps/acoustics_2d_homogeneous/acoustics.py (:6-92)
# --------------------------------------------------------------------------
def acoustics_homogeneous_setup(mx=100, my=100, split=True):
    x, dx = centers(-1.0, 1.0, mx)
    y, dy = centers(-1.0, 1.0, my)
    rho, bulk = 1.0, 4.0
    cc = np.sqrt(bulk / rho)
    zz = rho * cc
    q = np.empty((3, mx, my), order="F")
    Y, X = np.meshgrid(y, x)
    r = np.sqrt(X ** 2 + Y ** 2)
    width = 0.2
    q[0, :, :] = (np.abs(r - 0.5) <= width) * (1. + np.cos(np.pi * (r - 0.5) / width))
    q[1, :, :] = 0.
    q[2, :, :] = 0.
    p = _abi.make_problem(
        rp=_abi.RP_ACOUSTICS, num_eqn=3, num_waves=2, num_aux=0, mx=mx, my=my, dx=dx, dy=dy,
        order=2, transverse=-1 if split else 1, mthlim=[4],
        bc_lower=(_abi.BC_EXTRAP, _abi.BC_EXTRAP), bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP),
        params=(rho, bulk, cc, zz))
    cfl_desired = 0.45
    run = dict(cfl_max=0.5, cfl_desired=cfl_desired, dt_initial=np.min([dx, dy]) / cc * cfl_desired)
    return p, q, None, run


# --------------------------------------------------------------------------
# apps/acoustics_2d_variable/acoustics.py (:8-88)
# --------------------------------------------------------------------------
def acoustics_variable_setup(mx=200, my=200):
    x, dx = centers(-1.0, 1.0, mx)
    y, dy = centers(-1.0, 1.0, my)
    Y, X = np.meshgrid(y, x)
    rhol, rhor, bulkl, bulkr = 4.0, 1.0, 4.0, 4.0
    cl = np.sqrt(bulkl / rhol)
    cr = np.sqrt(bulkr / rhor)
    aux = np.empty((2, mx, my), order="F")
    aux[0, :, :] = rhol * (X < 0.) + rhor * (X >= 0.)
    aux[1, :, :] = cl * (X < 0.) + cr * (X >= 0.)
    x0, y0 = -0.5, 0.
    r = np.sqrt((X - x0) ** 2 + (Y - y0) ** 2)
    width, rad = 0.1, 0.25
    q = np.empty((3, mx, my), order="F")
    q[0, :, :] = (np.abs(r - rad) <= width) * (1. + np.cos(np.pi * (r - rad) / width))
    q[1, :, :] = 0.
    q[2, :, :] = 0.
    p = _abi.make_problem(
        rp=_abi.RP_VC_ACOUSTICS, num_eqn=3, num_waves=2, num_aux=2, mx=mx, my=my, dx=dx, dy=dy,
        order=2, transverse=1, mthlim=[4],
        bc_lower=(_abi.BC_WALL, _abi.BC_WALL), bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP),
        aux_bc_lower=(_abi.BC_WALL, _abi.BC_WALL), aux_bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP))
    run = dict(cfl_max=1.0, cfl_desired=0.9, dt_initial=0.1)
    return p, q, aux, run


def check_diff(expected, test, **kw):
    """src/pyclaw/util.py:149-167: returns None when within tolerance."""
    err_norm = np.linalg.norm(expected - test)
    expected_norm = np.linalg.norm(expected)
    test_norm = np.linalg.norm(test)
    if "abstol" in kw:
        return None if err_norm < kw["abstol"] else (expected_norm, test_norm, err_norm)
    if "reltol" in kw:
        return None if err_norm / expected_norm < kw["reltol"] else (expected_norm, test_norm, err_norm)
    raise Exception('Incorrect use of check_diff verifier, specify tol!')
