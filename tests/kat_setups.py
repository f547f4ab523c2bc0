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


# --------------------------------------------------------------------------
# apps/psystem_2d/psystem.py (:12-90 and psystem2D, :118-233; classic solver)
# --------------------------------------------------------------------------
PSYSTEM_GAUGES = [[0.25, 0.25], [17.85, 1.25], [3.25, 18.75], [11.75, 11.75]]


def psystem_setup():
    """Checkerboard of two nonlinear (exponential) materials, rho and E of 1
    and 4 in cells of 0.5; sigma(t=0) = 10 exp(-(x-0.25)^2 - (y-0.25)^2) at the
    walled corner; f-waves, superbee, unsplit with transverse_waves = 1 (the
    ClawSolver2D default), cfl 0.8/0.9, walls at the lower and extrapolation
    at the upper boundaries, t = 40 in 10 output intervals.  Returns (problem,
    q0, aux0 (aux[3] = q[0]), run settings, gauge cell indices)."""
    E1, p1, E2, p2 = 1., 1., 4., 4.
    x_lower, x_upper = 0.25, 20.25
    mx = my = int((x_upper - x_lower) * 10)
    x, dx = centers(x_lower, x_upper, mx)
    y, dy = centers(x_lower, x_upper, my)
    xfrac = x - np.floor(x / 1.0) * 1.0
    yfrac = y - np.floor(y / 1.0) * 1.0
    yyfrac, xxfrac = np.meshgrid(yfrac, xfrac)
    a = (xxfrac <= 0.5) * (yyfrac <= 0.5)
    b = (xxfrac > 0.5) * (yyfrac > 0.5)
    c = (xxfrac > 0.5) * (yyfrac <= 0.5)
    d = (xxfrac <= 0.5) * (yyfrac > 0.5)
    aux = np.empty((4, mx, my), order="F")
    aux[0] = p1 * a + p1 * b + p2 * c + p2 * d
    aux[1] = E1 * a + E1 * b + E2 * c + E2 * d
    aux[2] = 2 * a + 2 * b + 2 * c + 2 * d
    yy, xx = np.meshgrid(y, x)
    s = 10. * np.exp(-(xx - 0.25) ** 2 / (2 * 0.5) - (yy - 0.25) ** 2 / (2 * 0.5))
    q = np.empty((3, mx, my), order="F")
    q[0] = np.where(aux[2] == 1, 1, 0) * s / aux[1] + np.where(aux[2] == 2, 1, 0) * np.log(s + 1) / aux[1]
    q[1] = 0.
    q[2] = 0.
    aux[3] = q[0]
    p = _abi.make_problem(rp=_abi.RP_PSYSTEM, num_eqn=3, num_waves=2, num_aux=4, mx=mx, my=my, dx=dx, dy=dy,
                          order=2, transverse=1, mthlim=[2], use_fwave=True,
                          bc_lower=(_abi.BC_WALL, _abi.BC_WALL), bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP),
                          aux_bc_lower=(_abi.BC_WALL, _abi.BC_WALL),
                          aux_bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP))
    run = dict(cfl_max=0.9, cfl_desired=0.8, dt_initial=0.1)
    gauges = [[int(round((g[n] - x_lower) / dx)) for n in range(2)] for g in PSYSTEM_GAUGES]
    return p, q, aux, run, gauges


def psystem_gauge_values(q, aux):
    """gauge_pfunction of the app (:107-109): p = exp(eps E) - 1, and 10 p."""
    p = np.exp(q[0] * aux[1]) - 1
    return [p, 10 * p]


def psystem_oracle_run(orc, omp=True):
    """The app through the oracle: before every step aux[3] = q[0] (b4step,
    :86-90), gauges written at t = 0 and after every accepted step.  Returns
    the four gauges' (t, p, 10 p) rows and the final run."""
    p, q, aux, run, gauges = psystem_setup()
    rows = [[] for _ in gauges]

    def b4step(r):
        r.auxbc[3, 2:-2, 2:-2] = r.q[0]

    def record(r):
        for k, (ix, iy) in enumerate(gauges):
            rows[k].append([r.t] + psystem_gauge_values(r.q[:, ix, iy], r.auxbc[:, ix + 2, iy + 2]))

    r = orc.Run(p, q, aux, before_step=b4step, on_accept=record, omp=omp, **run)
    record(r)
    r.run(40.0, num_output_times=10, keep_copy=False)
    return [np.array(g) for g in rows], r
