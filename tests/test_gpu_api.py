"""GPU runs through the public pyclaw_b200 API (Controller.run /
ClawSolver2D.evolve_to_time), checked against the oracle's replay of the
reference driver loop and against the reference's own golden files."""
import os

import numpy as np
import pytest

import kat_setups as K
import pyclaw_b200 as pc

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _api_run(p, q, aux, run, tfinal, nout, split, trans=2, rp=None, bcs=None, src=None, keep=True,
             bounds=((0.0, 1.0), (0.0, 1.0)), before_step=None, outdir=None):
    """Build the same problem through the public API and run it on the GPU."""
    x = pc.Dimension('x', bounds[0][0], bounds[0][1], p.mx)
    y = pc.Dimension('y', bounds[1][0], bounds[1][1], p.my)
    assert x.delta == p.dx and y.delta == p.dy
    domain = pc.Domain([x, y])
    state = pc.State(domain, p.num_eqn, p.num_aux)
    state.q[...] = q
    if p.num_aux:
        state.aux[...] = aux
    solver = pc.ClawSolver2D(rp)
    names = {1: ('rho', 'bulk', 'cc', 'zz'), 3: ('gamma', 'gamma1'), 4: ('gamma', 'gamma1'), 5: ('grav',)}
    for k, key in enumerate(names.get(p.rp, ())):
        state.problem_data[key] = p.params[k]
    solver.dimensional_split = split
    solver.transverse_waves = trans
    solver.limiters = [int(p.mthlim[w]) for w in range(p.num_waves)]
    solver.bc_lower = [int(p.bc_lower[0]), int(p.bc_lower[1])]
    solver.bc_upper = [int(p.bc_upper[0]), int(p.bc_upper[1])]
    solver.aux_bc_lower = [int(p.aux_bc_lower[0]), int(p.aux_bc_lower[1])]
    solver.aux_bc_upper = [int(p.aux_bc_upper[0]), int(p.aux_bc_upper[1])]
    solver.cfl_max = run['cfl_max']
    solver.cfl_desired = run['cfl_desired']
    solver.dt_initial = run['dt_initial']
    if bcs:
        solver.user_bc_lower = bcs
    if src:
        solver.step_source = src
    if before_step is not None:
        solver.before_step = before_step
    claw = pc.Controller()
    claw.solution = pc.Solution(state, domain)
    claw.solver = solver
    claw.tfinal = tfinal
    claw.num_output_times = nout
    claw.output_format = None
    if outdir is not None:                      # the app's settings (acoustics.py:71-83)
        claw.output_format = 'ascii'
        claw.outdir = outdir
        claw.write_aux_init = True
    claw.keep_copy = keep
    claw.run()
    return claw, solver


def test_vc_acoustics_app_matches_golden_and_oracle(orc):
    """apps/acoustics_2d_variable: unsplit, trans=1, walls, rejected first step."""
    p, q, aux, run = K.acoustics_variable_setup()
    claw, solver = _api_run(p, q, aux, run, 0.6, 20, split=False, trans=1, rp=pc.riemann.rp2_vc_acoustics,
                            bounds=((-1.0, 1.0), (-1.0, 1.0)))
    ref = orc.Run(p, q, aux, omp=True, **run)
    frames = ref.run(0.6, num_output_times=20)
    got = claw.frames[20].state.q
    assert np.array_equal(got, frames[20])
    gold = np.load(os.path.join(GOLD, "vc_acoustics_pressure.npz"))["pressure"]
    assert np.max(np.abs(gold - got[0])) < 1e-13
    io = np.load(os.path.join(GOLD, "vc_acoustics_io.npz"))
    assert K.check_diff(io["q20"], got, reltol=1e-4) is None


def test_vc_acoustics_app_io_round_trip(tmp_path):
    """The reference's I/O test (apps/acoustics_2d_variable/
    test_acoustics_2d_variable_io.py:1-55): the app writes ascii frames through
    Controller.run while the device runs the steps; frames 0 (with aux) and 20
    are read back with Solution.read and compared with the reference's
    io_test_verification files at reltol 1e-4, and the header lines are the
    reference's text."""
    p, q, aux, run = K.acoustics_variable_setup()
    out = str(tmp_path / "_io_test_results")
    claw, solver = _api_run(p, q, aux, run, 0.6, 20, split=False, trans=1, rp=pc.riemann.rp2_vc_acoustics,
                            bounds=((-1.0, 1.0), (-1.0, 1.0)), outdir=out)
    assert sorted(f for f in os.listdir(out) if f.startswith("fort.q")) == ["fort.q%04d" % k for k in range(21)]
    io = np.load(os.path.join(GOLD, "vc_acoustics_io.npz"))
    s0 = pc.Solution(0, path=out, file_format='ascii', read_aux=True)
    s20 = pc.Solution(20, path=out, file_format='ascii', read_aux=False)
    assert K.check_diff(io["q20"], s20.state.q, reltol=1e-4) is None
    assert K.check_diff(io["aux0"], s0.state.aux, reltol=1e-4) is None
    with open(os.path.join(out, "fort.t0020")) as f:
        assert f.read() == str(io["t_header"])
    with open(os.path.join(out, "fort.q0020")) as f:
        assert "\n".join(f.read().splitlines()[:8]) == str(io["q_header"])
    # what was written is the device's frame at the %18.8e precision
    dev = claw.frames[20].state.q
    big = np.abs(dev) > 1e-300
    assert np.max(np.abs(s20.state.q[big] - dev[big]) / np.abs(dev[big])) <= 5.1e-9


def test_acoustics_homogeneous_split_app(orc):
    p, q, aux, run = K.acoustics_homogeneous_setup()
    claw, solver = _api_run(p, q, aux, run, 0.12, 10, split=True, rp=pc.riemann.rp2_acoustics,
                            bounds=((-1.0, 1.0), (-1.0, 1.0)))
    ref = orc.Run(p, q, aux, **run)
    frames = ref.run(0.12, num_output_times=10)
    got = claw.frames[-1].state.q
    assert np.array_equal(got, frames[-1])
    gold = np.load(os.path.join(GOLD, "acoustics_pressure.npz"))["pressure"]
    assert K.check_diff(gold, got[0], reltol=1e-3) is None


def test_shockbubble_app_custom_bc_and_source(orc):
    """apps/euler_2d/shockbubble.py: custom inflow BC and a Python source term run
    through the host-driven loop; abstol 1e-12 against the reference's file."""
    p, q, aux, run, bcs, src = K.shockbubble_setup()
    cb = bcs[(0, "lower")]

    def user_bc(state, dim, t, qbc, num_ghost):
        if dim.name == 'x':
            cb(qbc, t)

    def step_source(solver, state, dt):
        src(state.q, dt)

    claw, solver = _api_run(p, q, aux, run, 0.2, 1, split=True, rp=pc.riemann.rp2_euler_5wave,
                            bcs=user_bc, src=step_source, bounds=((0.0, 2.0), (0.0, 0.5)))
    got = claw.frames[1].state.q
    ref = orc.Run(p, q, aux, bc_callbacks=bcs, step_source=src, **run)
    frames = ref.run(0.2, num_output_times=1)
    assert np.array_equal(got, frames[1])
    gold = np.load(os.path.join(GOLD, "shockbubble_density.npz"))["density"]
    assert K.check_diff(0, np.linalg.norm(gold - got[0]), abstol=1e-12) is None


def _shockbubble_hooks():
    rinf, vinf, einf = K._shock_state()
    inflow = pc.hooks.FixedStateBC([rinf, rinf * vinf, 0., einf, 0.], side="lower")
    return inflow, pc.hooks.EulerRadialSource(radius_aux=0)


def test_shockbubble_app_on_the_device(orc):
    """The same app with its inflow condition and radial source given as the
    device-side hooks: the whole evolve_to_time loop stays on the GPU (source
    fused into the step kernel) and the result equals the oracle's run with
    the app's own Python callbacks, and the reference's file to 1e-12."""
    p, q, aux, run, bcs, src = K.shockbubble_setup()
    inflow, source = _shockbubble_hooks()
    claw, solver = _api_run(p, q, aux, run, 0.2, 1, split=True, rp=pc.riemann.rp2_euler_5wave,
                            bcs=inflow, src=source, bounds=((0.0, 2.0), (0.0, 0.5)))
    assert solver._device_loop_ok(claw.solution)
    got = claw.frames[1].state.q
    ref = orc.Run(p, q, aux, bc_callbacks=bcs, step_source=src, **run)
    frames = ref.run(0.2, num_output_times=1)
    assert np.array_equal(got, frames[1]), np.max(np.abs(got - frames[1]))
    assert solver.status['numsteps'] == ref.steps_taken
    gold = np.load(os.path.join(GOLD, "shockbubble_density.npz"))["density"]
    assert K.check_diff(0, np.linalg.norm(gold - got[0]), abstol=1e-12) is None


def test_shockbubble_hooks_on_the_host_path(orc):
    """The hook objects are ordinary callbacks too: with a before_step
    callback forcing the host-driven loop the result is the same."""
    p, q, aux, run, bcs, src = K.shockbubble_setup()
    inflow, source = _shockbubble_hooks()
    claw, solver = _api_run(p, q, aux, run, 0.2, 1, split=True, rp=pc.riemann.rp2_euler_5wave,
                            bcs=inflow, src=source, bounds=((0.0, 2.0), (0.0, 0.5)), before_step=lambda s, st: None)
    assert not solver._device_loop_ok(claw.solution)
    ref = orc.Run(p, q, aux, bc_callbacks=bcs, step_source=src, **run)
    frames = ref.run(0.2, num_output_times=1)
    assert np.array_equal(claw.frames[1].state.q, frames[1])


def test_config1_acoustics_full_run_parity(orc):
    """256x256 acoustics, walls, unsplit trans=2, MC, cfl 0.9, to t=0.6: the
    whole device-controlled run must equal the oracle cell for cell (the bar
    is 1e-11 relative; the result is identical), with the same dt sequence,
    and mass must be conserved to round-off."""
    import bench
    p, q, aux, run, tfinal = bench.acoustics_config()
    claw, solver = _api_run(p, q, aux, run, tfinal, 1, split=False, trans=2, rp=pc.riemann.rp2_acoustics,
                            bounds=((-1.0, 1.0), (-1.0, 1.0)))
    got = claw.solution.state.q
    ref = orc.Run(p, q, aux, omp=True, **run)
    ref.run(tfinal, num_output_times=1, keep_copy=False)
    rel = np.max(np.abs(got - ref.q)) / np.max(np.abs(ref.q))
    assert rel <= 1e-11, rel
    assert np.array_equal(got, ref.q)
    assert solver.status['numsteps'] == ref.steps_taken and claw.solution.t == ref.t
    mass0 = np.sum(q[0])
    assert abs(np.sum(got[0]) - mass0) <= 1e-12 * max(1.0, abs(mass0)) * p.mx


def test_config2_shockbubble_reduced_full_run(orc):
    """The shock-bubble workload at 320x80 (a quarter of the benchmark's
    resolution per axis) run to t=0.6: identical to the oracle."""
    import bench
    p, q, aux, run, tfinal = bench.shockbubble_config(320, 80)
    claw, solver = _api_run(p, q, aux, run, tfinal, 1, split=False, trans=2, rp=pc.riemann.rp2_euler_4wave,
                            bounds=((0.0, 2.0), (0.0, 0.5)))
    got = claw.solution.state.q
    ref = orc.Run(p, q, aux, omp=True, **run)
    ref.run(tfinal, num_output_times=1, keep_copy=False)
    assert np.array_equal(got, ref.q), np.max(np.abs(got - ref.q))
    assert solver.status['numsteps'] == ref.steps_taken


def test_config2_full_size_first_steps(orc):
    """1280x320 shock bubble: the first 12 device-controlled steps equal the oracle."""
    import bench
    p, q, aux, run, tfinal = bench.shockbubble_config()
    x = pc.Dimension('x', 0.0, 2.0, p.mx)
    y = pc.Dimension('y', 0.0, 0.5, p.my)
    domain = pc.Domain([x, y])
    state = pc.State(domain, 4)
    state.problem_data['gamma'] = 1.4
    state.problem_data['gamma1'] = 1.4 - 1.0
    state.q[...] = q
    solver = bench.make_solver(pc, p, run)
    sol = pc.Solution(state, domain)
    solver.setup(sol)
    solver.dt = run['dt_initial']
    ref = orc.Run(p, q, aux, omp=True, **run)
    for _ in range(12):
        solver.evolve_to_time(sol)          # one step (take_one_step)
        ref.evolve_to_time(None)
        assert solver.dt == ref.dt and sol.t == ref.t
    assert np.array_equal(sol.state.q, ref.q)


def test_config2_full_size_full_run(orc):
    """The benchmark workload itself: 1280x320 shock bubble run to t = 0.6
    (about 3000 controlled steps) by the device loop equals the oracle's C
    replay of evolve_to_time cell for cell (the bar is 1e-11 relative per
    cell), with the same number of steps and the same final time."""
    import ctypes
    import bench
    from pyclaw_b200 import _abi, _lib
    from pyclaw_b200.device import DeviceState
    p, q, aux, run, tfinal = bench.shockbubble_config()
    dev = DeviceState(p)
    dev.upload_q(q)
    c = _abi.Control()
    _lib.load().claw2_control_init(ctypes.byref(c), 0.0, run['dt_initial'], tfinal, run['cfl_max'],
                                   run['cfl_desired'], 1e99, 1, 0, 100000, run['cfl_desired'])
    out = dev.evolve(c)
    got = dev.download_q()
    assert out.error == 0 and abs(out.t - tfinal) == 0.0
    qbc = orc.new_qbc(p, q)
    ctrl = orc.control_init(0.0, run['dt_initial'], tfinal, run['cfl_max'], run['cfl_desired'], max_steps=100000)
    rc = orc.evolve(p, qbc, None, ctrl, omp=True)
    assert rc == 0, rc
    ref = np.array(qbc[:, 2:-2, 2:-2])
    for m in range(4):
        rel = np.max(np.abs(got[m] - ref[m])) / np.max(np.abs(ref[m]))
        assert rel <= 1e-11, (m, rel)
    assert np.array_equal(got, ref)
    assert out.numsteps == ctrl.numsteps and out.t == ctrl.t and out.rejected == ctrl.rejected


def test_walled_euler_conserves_mass_and_energy():
    import bench
    p, q, aux, run, tfinal = bench.shockbubble_config(320, 80, walls=True)
    claw, solver = _api_run(p, q, aux, run, 0.2, 1, split=False, trans=2, rp=pc.riemann.rp2_euler_4wave,
                            bounds=((0.0, 2.0), (0.0, 0.5)))
    got = claw.solution.state.q
    for m in (0, 3):
        s0, s1 = np.sum(q[m]), np.sum(got[m])
        assert abs(s1 - s0) <= 64 * np.finfo(float).eps * np.sum(np.abs(q[m])) * 10, (m, s1 - s0)


def test_walled_shallow_water_conserves_mass():
    """The dam break of config 3 at 192^2 with walls on every side, unsplit
    and split, through the public API: total depth is conserved to round-off."""
    import bench
    from pyclaw_b200 import _abi
    p, q, run = bench.shallow_config(192)
    for side in range(2):
        p.bc_lower[side] = _abi.BC_WALL
        p.bc_upper[side] = _abi.BC_WALL
    for split in (False, True):
        claw, solver = _api_run(p, q, None, run, 0.4, 1, split=split, trans=-1 if split else 2,
                                rp=pc.riemann.rp2_shallow_roe_with_efix, bounds=((-2.5, 2.5), (-2.5, 2.5)))
        got = claw.solution.state.q
        s0, s1 = np.sum(q[0]), np.sum(got[0])
        assert abs(s1 - s0) <= 64 * np.finfo(float).eps * s0 * 10, (split, s1 - s0)
        assert solver.status['numsteps'] > 10


def test_fixed_dt_too_large_gives_up():
    p, q, aux, run = K.acoustics_homogeneous_setup(mx=40, my=40, split=False)
    x = pc.Dimension('x', -1.0, 1.0, 40)
    y = pc.Dimension('y', -1.0, 1.0, 40)
    domain = pc.Domain([x, y])
    state = pc.State(domain, 3)
    state.problem_data.update(rho=1.0, bulk=4.0, cc=2.0, zz=2.0)
    state.q[...] = q
    solver = pc.ClawSolver2D(pc.riemann.rp2_acoustics)
    solver.dimensional_split = False
    solver.bc_lower = [pc.BC.extrap] * 2
    solver.bc_upper = [pc.BC.extrap] * 2
    solver.dt_variable = False
    solver.dt_initial = 0.1
    solver.dt = 0.1
    sol = pc.Solution(state, domain)
    with pytest.raises(Exception, match="CFL too large, giving up!"):
        solver.evolve_to_time(sol, 0.2)


def test_session_step2_host_buffers(orc):
    """The f2py-shaped entry point: reference-layout host arrays in and out."""
    import ctypes
    import gpu_helpers as H
    from pyclaw_b200 import _lib
    lib = _lib.load()
    p = H.problem("euler4", 45, 33, 2)
    q, _ = H.init_fields(p)
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    s = ctypes.c_void_p()
    _lib.check(lib.claw2_session_create(ctypes.byref(p), ctypes.byref(s)), "session_create")
    try:
        qnew = qbc.copy(order="F")
        cfl = ctypes.c_double()
        _lib.check(lib.claw2_session_step2(s, qbc.ctypes.data, qnew.ctypes.data, None, 0.003, ctypes.byref(cfl)),
                   "session_step2")
        ref = qbc.copy(order="F")
        cref = orc.step_hyperbolic(p, ref, None, 0.003)
        assert cfl.value == cref
        assert np.array_equal(qnew[:, 2:-2, 2:-2], ref[:, 2:-2, 2:-2])
    finally:
        lib.claw2_session_destroy(s)


def _gauged_vc_run(outdir, host_loop, orc=None):
    """apps/acoustics_2d_variable at 80x80 with four gauges (the psystem app's
    way of adding them, apps/psystem_2d/psystem.py:224-227) and a
    compute_gauge_values of q and aux, run to t = 0.4 through Controller.run."""
    p, q, aux, run = K.acoustics_variable_setup(mx=80, my=80)
    x = pc.Dimension('x', -1.0, 1.0, p.mx)
    y = pc.Dimension('y', -1.0, 1.0, p.my)
    domain = pc.Domain([x, y])
    state = pc.State(domain, 3, 2)
    state.q[...] = q
    state.aux[...] = aux
    state.keep_gauges = True
    state.grid.add_gauges([[-0.5, 0.0], [0.25, 0.3], [0.9, -0.9], [-0.95, 0.95]])
    solver = pc.ClawSolver2D(pc.riemann.rp2_vc_acoustics)
    solver.dimensional_split = False
    solver.transverse_waves = 1
    solver.limiters = pc.limiters.tvd.MC
    solver.bc_lower = [pc.BC.wall, pc.BC.wall]
    solver.bc_upper = [pc.BC.extrap, pc.BC.extrap]
    solver.aux_bc_lower = [pc.BC.wall, pc.BC.wall]
    solver.aux_bc_upper = [pc.BC.extrap, pc.BC.extrap]
    solver.dt_initial = run['dt_initial']
    solver.compute_gauge_values = lambda qg, ag: [qg[0] * ag[0], qg[1] + qg[2]]
    if host_loop:
        solver.before_step = lambda s, st: None           # forces the host-driven loop
    claw = pc.Controller()
    claw.solution = pc.Solution(state, domain)
    claw.solver = solver
    claw.outdir = outdir
    claw.output_format = None
    claw.tfinal = 0.4
    claw.num_output_times = 4
    claw.run()
    return claw, solver, state, (p, q, aux, run)


def test_gauges_recorded_on_the_device(orc, tmp_path):
    """Gauges keep the time loop on the device (samples recorded after every
    accepted step, drained after each batch of steps) and give exactly what
    write_gauge_values gives on the host-driven loop, in memory and in the
    gauge files; the last samples equal the oracle's final state."""
    claw_d, solver_d, st_d, (p, q, aux, run) = _gauged_vc_run(str(tmp_path / "dev"), host_loop=False)
    assert solver_d._device_loop_ok(claw_d.solution)
    claw_h, solver_h, st_h, _ = _gauged_vc_run(str(tmp_path / "host"), host_loop=True)
    assert not solver_h._device_loop_ok(claw_h.solution)
    assert len(st_d.gauge_data) == 4
    nsteps = solver_d.status['numsteps']
    for gd, gh in zip(st_d.gauge_data, st_h.gauge_data):
        assert gd.shape == gh.shape and gd.shape[0] >= 2
        assert np.array_equal(gd, gh)
    for name in st_d.grid.gauge_file_names:
        with open(os.path.join(str(tmp_path / "dev"), "_gauges", name)) as f:
            text_d = f.read()
        with open(os.path.join(str(tmp_path / "host"), "_gauges", name)) as f:
            text_h = f.read()
        assert text_d == text_h and len(text_d.splitlines()) >= nsteps
    ref = orc.Run(p, q, aux, **run)
    frames = ref.run(0.4, num_output_times=4)
    for i, (ix, iy) in enumerate(st_d.grid.gauges):
        qg = frames[-1][:, ix, iy]
        assert st_d.gauge_data[i][-1][0] == ref.t
        assert list(st_d.gauge_data[i][-1][1:]) == [qg[0] * aux[0, ix, iy], qg[1] + qg[2]]


def _psystem_api_run(before_step, outdir):
    """apps/psystem_2d/psystem.py:118-233 through the public API."""
    p, q, aux, run, gauges = K.psystem_setup()
    x = pc.Dimension('x', 0.25, 20.25, p.mx)
    y = pc.Dimension('y', 0.25, 20.25, p.my)
    domain = pc.Domain([x, y])
    state = pc.State(domain, 3, 4)
    state.aux[...] = aux
    state.q[...] = q
    state.keep_gauges = True
    state.grid.add_gauges(K.PSYSTEM_GAUGES)
    assert [list(g) for g in state.grid.gauges] == gauges
    solver = pc.ClawSolver2D(pc.riemann.rp2_psystem)
    solver.limiters = pc.limiters.tvd.superbee
    solver.bc_lower = [pc.BC.wall, pc.BC.wall]
    solver.bc_upper = [pc.BC.extrap, pc.BC.extrap]
    solver.aux_bc_lower = [pc.BC.wall, pc.BC.wall]
    solver.aux_bc_upper = [pc.BC.extrap, pc.BC.extrap]
    solver.fwave = True
    solver.cfl_max = 0.9
    solver.cfl_desired = 0.8
    solver.before_step = before_step
    solver.dimensional_split = False
    solver.compute_gauge_values = K.psystem_gauge_values
    claw = pc.Controller()
    claw.tfinal = 40.0
    claw.solver = solver
    claw.outdir = outdir
    claw.solution = pc.Solution(state, domain)
    claw.num_output_times = 10
    claw.output_format = None
    claw.run()
    return claw, solver, state


def test_psystem_fwave_app_matches_reference_gauges(orc, tmp_path):
    """apps/psystem_2d/test_2d_psystem.py on the GPU: the f-wave p-system with
    its before-step copy of eps into aux (hooks.AuxFromQ, a copy kernel
    before every step) and its four gauges (recorded on the device), the
    whole 40-time-unit run in the device loop.  Gauges against the
    reference's verify_gauge*.txt at its reltol 1e-4 (reached: 1e-10), against
    the oracle's run to 1e-11 relative (the solver calls exp, whose last bit
    may differ between the host's and the device's libraries), and the same
    app with the copy as a Python callback (host loop) is bit-identical."""
    claw, solver, state = _psystem_api_run(pc.hooks.AuxFromQ(3, 0), str(tmp_path / "dev"))
    assert solver._device_loop_ok(claw.solution)
    gold = np.load(os.path.join(GOLD, "psystem_gauges.npz"))
    rows, r = K.psystem_oracle_run(orc)
    for i, key in enumerate(("g0p25_0p25", "g17p85_1p25", "g3p25_18p75", "g11p75_11p75")):
        got = np.asarray(state.gauge_data[i])
        assert got.shape == gold[key].shape, (key, got.shape)
        assert K.check_diff(gold[key], got, reltol=1e-4) is None, key
        assert np.linalg.norm(gold[key] - got) / np.linalg.norm(gold[key]) < 1e-10, key
        assert np.max(np.abs(got - rows[i])) <= 1e-11 * np.max(np.abs(rows[i])), key
    scale = np.max(np.abs(r.q), axis=(1, 2))
    assert np.all(np.max(np.abs(state.q - r.q), axis=(1, 2)) <= 1e-11 * scale)

    def b4step(s, st):
        st.aux[3, :, :] = st.q[0, :, :]
    claw_h, solver_h, state_h = _psystem_api_run(b4step, str(tmp_path / "host"))
    assert not solver_h._device_loop_ok(claw_h.solution)
    for gd, gh in zip(state.gauge_data, state_h.gauge_data):
        assert np.array_equal(gd, gh)
    assert np.array_equal(state.q, state_h.q)


def test_session_evolve_host_buffers_matches_oracle(orc):
    """claw2_session_evolve, the host-buffer form of one Controller.run output
    interval (state up, the interval's steps under the device controller in
    batches sized by its own estimate, state down), over two intervals: the
    same state, t, dt and step count as the oracle's evolve_to_time."""
    import ctypes
    import gpu_helpers as H
    from pyclaw_b200 import _lib
    lib = _lib.load()
    p = H.problem("euler4", 97, 61, 2, bcl=(1, 3), bcu=(1, 3))
    q, _ = H.init_fields(p, seed=21)
    dt0 = 0.3 / 97
    ref = orc.Run(p, q, None, cfl_max=1.0, cfl_desired=0.9, dt_initial=dt0)
    s = ctypes.c_void_p()
    _lib.check(lib.claw2_session_create(ctypes.byref(p), ctypes.byref(s)), "session_create")
    try:
        host = np.asfortranarray(q.copy())
        t = ctypes.c_double(0.0)
        dt = ctypes.c_double(dt0)
        status = (ctypes.c_double * 5)()
        steps = 0
        for tend in (0.05, 0.12):
            _lib.check(lib.claw2_session_evolve(s, host.ctypes.data, None, ctypes.byref(t), ctypes.byref(dt), tend,
                                                1.0, 0.9, 1e99, 100000, status), "session_evolve")
            steps += int(status[3])
            ref.evolve_to_time(tend)
            assert t.value == ref.t == tend
            assert np.array_equal(host, ref.q)
        assert dt.value == ref.dt
        assert steps == ref.steps_taken and steps > 40
    finally:
        lib.claw2_session_destroy(s)
