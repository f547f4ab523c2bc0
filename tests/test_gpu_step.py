"""GPU parity of the sm_100a step against the CPU oracle, through the C ABI.

Every case advances the same ghost-filled state with libclaw2.so's claw2_step
and with the oracle's restatement of step2/step2ds, and requires the interior
to be identical (==, so only the sign of exact zeros may differ), the CFL
number to be identical, and the ghost cells the kernel writes for the next
step to equal the reference boundary fill of the new state.
"""
import itertools

import numpy as np
import pytest

import gpu_helpers as H

pytestmark = pytest.mark.gpu

G = 2
I = np.s_[:, G:-G, G:-G]

CASES = []
for name, tr in itertools.product(["acoustics", "vc_acoustics", "euler4", "euler5", "shallow"], [2, 1, 0, -1]):
    CASES.append((name, 61, 47, tr, 2, (1, 3), (1, 3)))
CASES += [
    ("euler4", 29, 29, 2, 2, (1, 3), (1, 3)),      # exactly one unsplit tile
    ("euler4", 30, 58, 2, 2, (3, 3), (3, 3)),      # partial tiles, all walls
    ("euler4", 28, 28, -1, 2, (1, 1), (1, 1)),     # exactly one split tile
    ("acoustics", 57, 33, 2, 1, (2, 2), (2, 2)),   # first order, periodic
    ("shallow", 64, 64, 2, 2, (2, 3), (2, 3)),     # periodic x, walls y
    ("vc_acoustics", 4, 4, 2, 2, (3, 3), (1, 1)),  # smallest grid with fused ghosts
    ("euler5", 3, 2, 2, 2, (1, 1), (1, 1)),        # tiny grid: separate ghost fill
    ("euler4", 300, 7, 2, 2, (1, 3), (1, 3)),      # long and thin
    ("euler4", 7, 300, -1, 2, (1, 3), (1, 3)),
    # grids of at least 148 29x29 tiles: the acoustics bodies' large-tile form
    # (smaller grids run 13x13 tiles)
    ("vc_acoustics", 400, 380, 2, 2, (1, 3), (3, 1)),
    ("acoustics", 420, 360, 1, 2, (3, 2), (3, 2)),
]


@pytest.mark.parametrize("name,mx,my,tr,order,bcl,bcu", CASES)
def test_step_bit_identical_to_oracle(orc, name, mx, my, tr, order, bcl, bcu):
    lim = (4,) if name not in ("euler5",) else (4, 4, 4, 4, 2)
    p = H.problem(name, mx, my, tr, order=order, mthlim=lim, bcl=bcl, bcu=bcu)
    q, aux = H.init_fields(p, seed=mx * 7 + my)
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    auxbc = None
    if p.num_aux:
        auxbc = orc.new_qbc(p, aux, p.num_aux)
        orc.fill_aux_ghosts(p, auxbc)
    dt = 0.25 / max(mx, my)
    ref = qbc.copy(order="F")
    cfl_ref = orc.step_hyperbolic(p, ref, auxbc, dt)
    out, cfl = H.dev_step(p, qbc, auxbc, dt)
    assert np.array_equal(out[I], ref[I]), np.nanmax(np.abs(out[I] - ref[I]))
    assert cfl == cfl_ref
    orc.fill_ghosts(p, ref)
    assert np.array_equal(out, ref), "ghost cells differ from the boundary fill of the new state"


LIMITER_CASES = [(name, lim, order, tr) for name in ("euler4", "shallow") for lim in (0, 1, 2, 3, 5)
                 for order, tr in ((2, 2), (2, 1))]
LIMITER_CASES += [("euler4", 4, 1, 2), ("shallow", 2, 1, 1), ("euler5", 2, 2, 2), ("euler5", 1, 1, 0)]


@pytest.mark.parametrize("name,lim,order,tr", LIMITER_CASES)
def test_unsplit_limiters_bit_identical_to_oracle(orc, name, lim, order, tr):
    """Every limiter id (0 = none, 1-5) and first order through the unsplit
    bodies of the dense-wave solvers, on a grid of several partial tiles."""
    mx, my = 75, 62
    p = H.problem(name, mx, my, tr, order=order, mthlim=(lim,), bcl=(1, 3), bcu=(3, 1))
    q, aux = H.init_fields(p, seed=lim * 13 + order + tr)
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    dt = 0.25 / max(mx, my)
    ref = qbc.copy(order="F")
    cfl_ref = orc.step_hyperbolic(p, ref, None, dt)
    out, cfl = H.dev_step(p, qbc, None, dt)
    assert np.array_equal(out[I], ref[I]), np.nanmax(np.abs(out[I] - ref[I]))
    assert cfl == cfl_ref
    orc.fill_ghosts(p, ref)
    assert np.array_equal(out, ref)


CAPA_FWAVE_CASES = [("vc_acoustics", capa, fw, tr) for capa in (-1, 0, 1) for fw in (0, 1) for tr in (2, 1, 0, -1)
                    if capa >= 0 or fw]
CAPA_FWAVE_CASES += [("acoustics", -1, 1, tr) for tr in (2, -1)] + [("euler4", -1, 1, 2), ("shallow", -1, 1, -1)]


@pytest.mark.parametrize("name,capa,fwave,tr", CAPA_FWAVE_CASES)
def test_capacity_and_fwave_branches_bit_identical_to_oracle(orc, name, capa, fwave, tr):
    """The capacity-function branch (dtdx/kappa per cell, the update divided by
    kappa; step2.f90:101-105,151-163, flux2.f90) and the f-wave branch of the
    second-order correction (sign(s) for |s|, flux2.f90:150-162) through the
    generic tile body, against the oracle.  The solvers here are not f-wave
    solvers and aux component `capa` is not a physical capacity; the cases
    exercise the branches' arithmetic, which must agree exactly."""
    mx, my = 61, 47
    p = H.problem(name, mx, my, tr, bcl=(1, 3), bcu=(3, 1))
    p.index_capa = capa
    p.use_fwave = fwave
    q, aux = H.init_fields(p, seed=capa * 5 + fwave * 3 + tr + 17)
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    auxbc = None
    if p.num_aux:
        auxbc = orc.new_qbc(p, aux, p.num_aux)
        orc.fill_aux_ghosts(p, auxbc)
    dt = 0.25 / max(mx, my)
    ref = qbc.copy(order="F")
    cfl_ref = orc.step_hyperbolic(p, ref, auxbc, dt)
    out, cfl = H.dev_step(p, qbc, auxbc, dt)
    assert np.array_equal(out[I], ref[I]), np.nanmax(np.abs(out[I] - ref[I]))
    assert cfl == cfl_ref
    orc.fill_ghosts(p, ref)
    assert np.array_equal(out, ref)


def _random_cases(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        name = ["acoustics", "vc_acoustics", "euler4", "euler5", "shallow"][int(rng.integers(0, 5))]
        mx, my = (int(v) for v in rng.integers(1, 90, 2))
        tr = int(rng.choice([2, 1, 0, -1]))
        bcl = tuple(int(v) for v in rng.choice([1, 2, 3], 2))
        bcu = tuple(b if b == 2 else int(rng.choice([1, 3])) for b in bcl)   # periodic sides pair up
        lim = int(rng.integers(0, 6))
        order = int(rng.choice([1, 2]))
        out.append((name, mx, my, tr, order, lim, bcl, bcu))
    return out


@pytest.mark.parametrize("name,mx,my,tr,order,lim,bcl,bcu", _random_cases(40, 2026))
def test_random_configurations_bit_identical_to_oracle(orc, name, mx, my, tr, order, lim, bcl, bcu):
    """Seeded random solver, grid size (1..89 cells a side, so single cells,
    thin strips and partial tiles of every body), transverse mode, order,
    limiter and boundary conditions: one step equals the oracle's."""
    p = H.problem(name, mx, my, tr, order=order, mthlim=(lim,), bcl=bcl, bcu=bcu)
    q, aux = H.init_fields(p, seed=mx * 131 + my)
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    auxbc = None
    if p.num_aux:
        auxbc = orc.new_qbc(p, aux, p.num_aux)
        orc.fill_aux_ghosts(p, auxbc)
    dt = 0.2 / max(mx, my)
    ref = qbc.copy(order="F")
    cfl_ref = orc.step_hyperbolic(p, ref, auxbc, dt)
    out, cfl = H.dev_step(p, qbc, auxbc, dt)
    assert np.array_equal(out[I], ref[I]), np.nanmax(np.abs(out[I] - ref[I]))
    assert cfl == cfl_ref
    orc.fill_ghosts(p, ref)
    assert np.array_equal(out, ref)


def test_nonfinite_state_is_reported(orc):
    p = H.problem("euler4", 40, 40, 2)
    q, _ = H.init_fields(p)
    q[0, 10, 10] = -1.0                      # negative density -> sqrt of a negative number
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    out, cfl = H.dev_step(p, qbc, None, 0.001)
    assert np.isnan(cfl)
    # the context is still usable afterwards
    q2, _ = H.init_fields(p, seed=3)
    qbc2 = orc.new_qbc(p, q2)
    orc.fill_ghosts(p, qbc2)
    ref = qbc2.copy(order="F")
    cfl_ref = orc.step_hyperbolic(p, ref, None, 0.001)
    out2, cfl2 = H.dev_step(p, qbc2, None, 0.001)
    assert cfl2 == cfl_ref and np.array_equal(out2[I], ref[I])


def test_repeated_steps_are_deterministic():
    p = H.problem("euler4", 90, 70, 2)
    q, _ = H.init_fields(p)
    from oracle import oracle as O
    qbc = O.new_qbc(p, q)
    O.fill_ghosts(p, qbc)
    a, ca = H.dev_step(p, qbc, None, 0.002)
    b, cb = H.dev_step(p, qbc, None, 0.002)
    assert ca == cb and np.array_equal(a, b)


def test_halo_wait_runs_out_and_reports_timeout(orc):
    """The TMA-staged lean body waits on an mbarrier for its halo copies with a
    limit of about a second.  Making every CTA wait for 8 bytes more than its
    copies deliver (a count that nothing completes) must end the step with
    CLAW2_ERR_TIMEOUT through the controller, or a NaN CFL number without one,
    and leave the context usable: the next run is bit-identical to the oracle."""
    import ctypes
    import torch
    from pyclaw_b200 import _abi, _lib
    from pyclaw_b200.device import DeviceState
    lib = _lib.load()
    p = H.problem("euler4", 60, 40, 2, bcl=(1, 3), bcu=(1, 3))
    q, _ = H.init_fields(p, seed=5)

    def controlled():
        dev = DeviceState(p)
        dev.upload_q(q)
        c = _abi.Control()
        _lib.check(lib.claw2_control_init(ctypes.byref(c), 0.0, 0.002, 0.01, 1.0, 0.9, 1e99, 1, 0, 100, 0.9),
                   "claw2_control_init")
        out = dev.evolve(c)
        return out, dev.download_q()

    try:
        _lib.check(lib.claw2_debug_halo_shortfall(8), "claw2_debug_halo_shortfall")
        out, _ = controlled()
        assert out.error == _abi.ERR_TIMEOUT and out.numsteps == 0, (out.error, out.numsteps)
        qbc = orc.new_qbc(p, q)
        orc.fill_ghosts(p, qbc)
        _, cfl = H.dev_step(p, qbc, None, 0.002)
        assert cfl != cfl                       # NaN: the step did not happen
    finally:
        lib.claw2_debug_halo_shortfall(0)
    torch.cuda.synchronize()
    out, got = controlled()
    assert out.error == 0 and out.numsteps > 0
    ref = orc.Run(p, q, None, cfl_max=1.0, cfl_desired=0.9, dt_initial=0.002)
    ref.evolve_to_time(0.01)
    assert np.array_equal(got, ref.q) and ref.steps_taken == out.numsteps


def _piecewise_uniform(p, kind, seed):
    """Fields made of uniform regions: a background state, a second uniform
    state over x >= 0.6 (its edge is a straight discontinuity), a noisy patch,
    and for kind 'still' a zero-velocity background (wall ghosts then mirror
    it exactly)."""
    rng = np.random.default_rng(seed)
    mx, my = p.mx, p.my
    x = (np.arange(mx) + 0.5) / mx
    y = (np.arange(my) + 0.5) / my
    X, Y = np.meshgrid(x, y, indexing='ij')
    right = X >= 0.6
    patch = (np.abs(X - 0.25) < 0.12) & (np.abs(Y - 0.4) < 0.15)
    noise = rng.random((mx, my))
    q = np.empty((p.num_eqn, mx, my), order='F')
    u0, v0 = (0.0, 0.0) if kind == "still" else (0.3, -0.2)
    if p.rp in (_abi.RP_EULER_4WAVE, _abi.RP_EULER_5WAVE):
        rho = np.where(right, 0.5, 1.0) + patch * 0.3 * noise
        u = np.where(right, u0 - 0.1, u0) + patch * 0.1 * noise
        v = np.full((mx, my), v0)
        pr = np.where(right, 0.7, 1.0) + patch * 0.2 * noise
        q[0] = rho
        q[1] = rho * u
        q[2] = rho * v
        q[3] = pr / 0.4 + 0.5 * rho * (u * u + v * v)
        if p.num_eqn == 5:
            q[4] = right * 1.0
    else:
        h = np.where(right, 1.5, 1.0) + patch * 0.2 * noise
        q[0] = h
        q[1] = h * (u0 + patch * 0.1 * noise)
        q[2] = h * v0
    return q


from pyclaw_b200 import _abi  # noqa: E402

UNIFORM_CASES = [
    ("euler4", 2, (1, 1), (1, 1), "moving", 150, 90),
    ("euler4", 1, (1, 3), (3, 1), "moving", 150, 90),
    ("euler4", 0, (3, 3), (3, 3), "still", 150, 90),
    ("euler4", 2, (3, 3), (3, 3), "still", 57, 85),      # partial tiles on both axes
    ("euler4", 2, (2, 1), (2, 1), "moving", 112, 56),    # periodic x: 4 x 2 full tiles
    ("euler5", 2, (1, 3), (1, 3), "moving", 150, 90),
    ("shallow", 2, (1, 1), (1, 1), "moving", 150, 90),
    ("shallow", 2, (3, 3), (3, 3), "still", 130, 70),
    ("shallow", 1, (1, 2), (1, 2), "moving", 100, 100),
    # more than 8 x 148 tiles: the lean body's 256-thread form (the grids
    # above run its 512-thread form)
    ("euler4", 2, (1, 3), (3, 1), "moving", 1000, 980),
    ("shallow", 2, (3, 3), (3, 3), "still", 1010, 1000),
    # dimensional splitting: the generic body (28x28 tiles) on the same data
    ("euler4", -1, (1, 3), (3, 1), "moving", 150, 90),
    ("euler5", -1, (2, 1), (2, 1), "moving", 112, 56),
    ("shallow", -1, (3, 3), (3, 3), "still", 130, 70),
    ("shallow", -1, (1, 1), (1, 1), "moving", 57, 85),
]


@pytest.mark.parametrize("name,tr,bcl,bcu,kind,mx,my", UNIFORM_CASES)
def test_uniform_tiles_bit_identical_to_oracle(orc, name, tr, bcl, bcu, kind, mx, my):
    """Tiles whose whole input halo holds one state take the lean body's short
    path (cells kept, CFL from one solve per direction); next to them tiles
    that straddle a discontinuity or the noisy patch take the full step.
    Three steps in a row, each compared with the oracle (values, CFL, ghost
    cells), so tiles change kind as the disturbance spreads."""
    p = H.problem(name, mx, my, tr, bcl=bcl, bcu=bcu)
    q = _piecewise_uniform(p, kind, seed=mx + my + tr)
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    dt = 0.2 / max(mx, my)
    for _ in range(3):
        ref = qbc.copy(order="F")
        cfl_ref = orc.step_hyperbolic(p, ref, None, dt)
        out, cfl = H.dev_step(p, qbc, None, dt)
        assert np.array_equal(out[I], ref[I]), np.nanmax(np.abs(out[I] - ref[I]))
        assert cfl == cfl_ref, (cfl, cfl_ref)
        orc.fill_ghosts(p, ref)
        assert np.array_equal(out, ref), "ghost cells differ from the boundary fill of the new state"
        qbc = np.asfortranarray(ref)


@pytest.mark.parametrize("name", ["euler4", "shallow"])
def test_all_uniform_grid_keeps_its_state_and_cfl(orc, name):
    """A grid holding one state everywhere: every tile takes the short path;
    the state is unchanged and the CFL number equals the oracle's."""
    p = H.problem(name, 97, 61, 2, bcl=(1, 1), bcu=(1, 1))
    q = _piecewise_uniform(p, "moving", seed=1)
    q[:] = q[:, :1, :1]
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    dt = 0.3 / 97
    ref = qbc.copy(order="F")
    cfl_ref = orc.step_hyperbolic(p, ref, None, dt)
    out, cfl = H.dev_step(p, qbc, None, dt)
    assert np.array_equal(out, ref) and np.array_equal(out[I], qbc[I])
    assert cfl == cfl_ref and cfl > 0.0



@pytest.mark.parametrize("name,mx,my,tr", [("euler4", 140, 84, 2), ("shallow", 1010, 1000, 2),
                                          ("acoustics", 120, 90, 2), ("vc_acoustics", 500, 460, 2),
                                          ("euler4", 140, 84, -1)])
def test_chained_steps_equal_single_step_calls(name, mx, my, tr):
    """claw2_advance launches each step after its first as a programmatic
    dependent of the step before (lean, light and generic bodies); 30 steps in
    one call must leave the state, t and dt bit for bit where 30 calls of one
    step do."""
    import ctypes
    from pyclaw_b200 import _abi, _lib
    from pyclaw_b200.device import DeviceState
    t = H.torch()
    lib = _lib.load()
    p = H.problem(name, mx, my, tr, bcl=(1, 3), bcu=(3, 1))
    if p.rp in (_abi.RP_ACOUSTICS, _abi.RP_VC_ACOUSTICS):
        q, aux = H.init_fields(p, seed=9)
    else:
        q, aux = _piecewise_uniform(p, "moving", seed=9), None
    results = []
    for calls in (1, 30):
        dev = DeviceState(p)
        if aux is not None:
            dev.upload_aux(aux)
        dev.upload_q(q)
        c = _abi.Control.from_address(dev.ctrl_host.data_ptr())
        _lib.check(lib.claw2_control_init(ctypes.byref(c), 0.0, 0.2 / max(mx, my), 1e9, 1.0, 0.9, 1e99, 1, 0,
                                          1 << 40, 0.9), "claw2_control_init")
        dev.ctrl.copy_(dev.ctrl_host)
        for _ in range(calls):
            _lib.check(lib.claw2_advance(ctypes.byref(p), dev.ptr(dev.q[0]), dev.ptr(dev.q[1]), dev.ptr(dev.aux),
                                         dev.ptr(dev.ctrl), dev.ptr(dev.scratch), 30 // calls, dev.stream),
                       "claw2_advance")
        t.cuda.synchronize()
        dev.ctrl_host.copy_(dev.ctrl)
        t.cuda.synchronize()
        c = _abi.Control.from_address(dev.ctrl_host.data_ptr())
        assert c.numsteps == 30 and c.error == 0
        dev.cur = c.cur
        results.append((dev.download_q(), c.t, c.dt))
    (qa, ta, da), (qb, tb, db) = results
    assert ta == tb and da == db
    assert np.array_equal(qa, qb)
