"""Parity at the benchmark sizes of the shallow-water and batched workloads.

Shallow water, 4096^2 radial dam break, 500 controlled steps (Roe with the
transonic fix, superbee, unsplit with transverse_waves=2, extrapolation BCs):
the device run of the whole grid is compared with the oracle's replay of
evolve_to_time (src/pyclaw/solver.py:632-691 around step2.f90:92-248) on the
central 2048^2 cells.  That is exact, not an approximation, under a condition
the test checks on the GPU after every step: every cell outside the central
block still holds the initial state (h = 1, hu = hv = 0).  Then

  - a cell outside the block only ever sees that constant state in its
    stencil, whose Riemann problems have zero waves, so it stays constant
    (up to the sign of an exact zero, which never changes a non-zero value);
  - the oracle's extrapolation ghost cells around the block are copies of
    its constant border, which are the values the block's neighbours hold in
    the full grid, so every cell of the block has the same inputs;
  - the CFL number is the same: constant-state interfaces contribute
    dt/dx * 1 in both runs, and the rest are the block's own interfaces.

So the block evolves exactly as in the full grid, the dt sequence is the same,
and the comparison is cell for cell (the bar is 1e-11 relative per cell).  The
disturbance (the numerical precursor ahead of the bore) spreads one cell per
step along each axis, from 410 cells off the centre to about 910 at step 500;
the block's half-width is 1024.  Total depth is also checked for conservation with walls on every
side at the full size.

Batched variable-coefficient acoustics: the full 1024-instance draw of the
benchmark (nx, ny ~ U{64..384}, 300 controlled steps each): every instance
equals its own plain-step run, and 8 instances equal the oracle.
"""
import ctypes

import numpy as np
import pytest

import bench
from pyclaw_b200 import _abi, _lib

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

N_FULL, STEPS, BLOCK = 4096, 500, 2048


def _shallow_device_run(p, q, run, nsteps, watch_block=None):
    """nsteps controlled steps of the whole grid on the device.  With
    watch_block = (off, n), after every step both state buffers are checked
    to hold the initial constant state outside rows/columns off..off+n-1."""
    import torch
    from pyclaw_b200.device import DeviceState
    lib = _lib.load()
    dev = DeviceState(p)
    dev.upload_q(q)
    dev.q[1].copy_(dev.q[0])
    c = _abi.Control()
    _lib.check(lib.claw2_control_init(ctypes.byref(c), 0.0, run["dt_initial"], 1e9, run["cfl_max"],
                                      run["cfl_desired"], 1e99, 1, 0, nsteps, run["cfl_desired"]),
               "claw2_control_init")
    host = _abi.Control.from_address(dev.ctrl_host.data_ptr())
    ctypes.memmove(ctypes.addressof(host), ctypes.addressof(c), ctypes.sizeof(c))
    dev.ctrl.copy_(dev.ctrl_host)
    bad = torch.zeros((), dtype=torch.bool, device=dev.device)
    for _ in range(nsteps):
        _lib.check(lib.claw2_advance(ctypes.byref(p), dev.ptr(dev.q[0]), dev.ptr(dev.q[1]), dev.ptr(dev.aux),
                                     dev.ptr(dev.ctrl), dev.ptr(dev.scratch), 1, dev.stream), "claw2_advance")
        if watch_block is not None:
            off, n = watch_block
            for k in (0, 1):
                v = dev.interior(k)
                for band in (v[:, :off, :], v[:, off + n:, :], v[:, off:off + n, :off], v[:, off:off + n, off + n:]):
                    bad |= (band[0] != 1.0).any() | (band[1] != 0.0).any() | (band[2] != 0.0).any()
    dev.ctrl_host.copy_(dev.ctrl)
    torch.cuda.synchronize()
    out = _abi.Control()
    ctypes.memmove(ctypes.addressof(out), ctypes.addressof(host), ctypes.sizeof(out))
    dev.cur = out.cur
    return dev, out, bool(bad.item())


def test_config3_shallow_4096_500_steps_matches_oracle(orc):
    p, q, run = bench.shallow_config(N_FULL)
    off = (N_FULL - BLOCK) // 2
    dev, out, spread = _shallow_device_run(p, q, run, STEPS, watch_block=(off, BLOCK))
    assert not spread, "the disturbance left the central %d^2 block; enlarge it" % BLOCK
    assert out.iter == STEPS and out.error in (0, _abi.ERR_MAX_STEPS)
    got = dev.download_q()
    del dev
    # outside the block the final state is the initial one
    assert np.all(got[0, :off, :] == 1.0) and np.all(got[0, off + BLOCK:, :] == 1.0)
    assert np.all(got[1:, :off, :] == 0.0) and np.all(got[1:, off + BLOCK:, :] == 0.0)

    pb = _abi.Problem.from_buffer_copy(p)
    pb.mx = pb.my = BLOCK
    qb = np.asfortranarray(q[:, off:off + BLOCK, off:off + BLOCK])
    qbc = orc.new_qbc(pb, qb)
    ctrl = orc.control_init(0.0, run["dt_initial"], 1e9, run["cfl_max"], run["cfl_desired"], max_steps=STEPS)
    rc = orc.evolve(pb, qbc, None, ctrl, omp=True)
    assert rc in (0, _abi.ERR_MAX_STEPS), rc
    ref = qbc[:, 2:-2, 2:-2]
    # the oracle's block kept its border constant too (same condition, seen from the oracle)
    assert np.all(ref[0, :2, :] == 1.0) and np.all(ref[0, -2:, :] == 1.0)
    blk = got[:, off:off + BLOCK, off:off + BLOCK]
    for m in range(3):
        scale = max(np.max(np.abs(ref[m])), np.finfo(float).tiny)
        rel = np.max(np.abs(blk[m] - ref[m])) / scale
        assert rel <= 1e-11, (m, rel)
    assert np.array_equal(blk, ref)
    assert out.numsteps == ctrl.numsteps and out.t == ctrl.t and out.dt == ctrl.dt
    assert out.rejected == ctrl.rejected


def test_config3_shallow_4096_walls_conserves_depth():
    """The same dam break with walls on every side, 500 steps at full size:
    total depth is conserved to round-off (a few ulp per cell-update of the
    sum's magnitude)."""
    p, q, run = bench.shallow_config(N_FULL)
    for side in range(2):
        p.bc_lower[side] = _abi.BC_WALL
        p.bc_upper[side] = _abi.BC_WALL
    dev, out, _ = _shallow_device_run(p, q, run, STEPS)
    assert out.iter == STEPS and out.numsteps > 0
    got = dev.download_q()
    s0, s1 = np.sum(q[0]), np.sum(got[0])
    assert abs(s1 - s0) <= 64 * np.finfo(float).eps * s0 * 10, s1 - s0
    assert np.all(np.isfinite(got))


def test_config4_all_1024_instances_equal_single_runs(orc):
    """The benchmark's batch: 1024 instances drawn as in bench.batched_vc_config
    (nx, ny ~ U{64..384}, 2-6 layers of rho, K ~ U[1,4], a Gaussian pulse),
    300 controlled steps of every instance in the persistent batched kernel
    replayed from CUDA graphs with the autotuned launch; each instance equals
    the plain device step run on it alone, and 8 instances spread over the
    batch equal the oracle's replay of evolve_to_time."""
    import torch
    from pyclaw_b200.batch import BatchSolver
    from pyclaw_b200.device import DeviceState
    nsteps = 300
    prob, insts = bench.batched_vc_config()
    bs = BatchSolver(prob, insts)
    bs.autotune(steps=2, repeats=1)
    bs.init_controls([i["dt"] for i in insts], max_steps=nsteps)
    bs.advance_graph(nsteps, chunk=50)
    ctrls = bs.controls()
    assert all(c.done and c.numsteps == nsteps for c in ctrls)
    lib = _lib.load()
    for k, inst in enumerate(insts):
        pk = bs.problems[k]
        dev = DeviceState(pk)
        dev.upload_aux(inst["aux"])
        dev.upload_q(inst["q"])
        c = _abi.Control()
        lib.claw2_control_init(ctypes.byref(c), 0.0, inst["dt"], 1e300, 1.0, 0.9, 1e99, 1, 0, nsteps, 0.9)
        alone = dev.evolve(c)
        assert alone.numsteps == ctrls[k].numsteps and alone.t == ctrls[k].t and alone.dt == ctrls[k].dt, k
        assert np.array_equal(dev.download_q(), bs.solution(k)), k
        del dev
    torch.cuda.synchronize()
    for k in np.linspace(0, len(insts) - 1, 8).round().astype(int):
        pk = bs.problems[k]
        ref = orc.Run(pk, insts[k]["q"], insts[k]["aux"], cfl_max=1.0, cfl_desired=0.9,
                      dt_initial=insts[k]["dt"], max_steps=nsteps, omp=True)
        try:
            ref.evolve_to_time(1e300)
        except Exception as e:               # nsteps iterations reached before tend, as configured
            assert "Maximum number of timesteps" in str(e)
        assert np.array_equal(bs.solution(k), ref.q), k
        assert ref.steps_taken == ctrls[k].numsteps
    bs.close()
