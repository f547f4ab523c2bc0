"""Batched form: every instance of a batch must be bit-identical to the same
instance stepped alone by the plain device path, whatever launch variant the
autotuner picks, and one instance is checked against the oracle."""
import ctypes

import numpy as np
import pytest

import bench
from pyclaw_b200 import _abi, _lib

pytestmark = pytest.mark.gpu


def _alone(prob, inst, nsteps):
    """The instance run by itself: DeviceState + the device-controlled loop."""
    import torch
    from pyclaw_b200.device import DeviceState
    pk = _abi.Problem.from_buffer_copy(prob)
    pk.mx, pk.my = inst["q"].shape[1], inst["q"].shape[2]
    pk.dx, pk.dy = inst["dx"], inst["dy"]
    dev = DeviceState(pk)
    dev.upload_aux(inst["aux"])
    dev.upload_q(inst["q"])
    lib = _lib.load()
    c = _abi.Control()
    lib.claw2_control_init(ctypes.byref(c), 0.0, inst["dt"], 1e300, 1.0, 0.9, 1e99, 1, 0, nsteps, 0.9)
    out = dev.evolve(c)
    torch.cuda.synchronize()
    return dev.download_q(), out


def test_batch_instances_equal_single_runs(orc):
    prob, insts = bench.batched_vc_config(n=12, seed=7, nmin=20, nmax=90)
    from pyclaw_b200.batch import BatchSolver
    bs = BatchSolver(prob, insts)
    bs.init_controls([i["dt"] for i in insts], max_steps=40)
    tuning = bs.autotune(steps=2, repeats=1)
    assert tuning["chosen"] in tuning["candidates"]
    bs.advance_graph(45, chunk=20)           # more launches than needed: done instances idle
    ctrls = bs.controls()
    for k in (0, 3, 7, 11):
        q_alone, c_alone = _alone(prob, insts[k], 40)
        assert ctrls[k].numsteps == c_alone.numsteps and ctrls[k].t == c_alone.t and ctrls[k].dt == c_alone.dt
        assert np.array_equal(bs.solution(k), q_alone)
    # one instance against the oracle's replay of evolve_to_time
    k = 5
    pk = bs.problems[k]
    ref = orc.Run(pk, insts[k]["q"], insts[k]["aux"], cfl_max=1.0, cfl_desired=0.9, dt_initial=insts[k]["dt"],
                  max_steps=40)
    try:
        ref.evolve_to_time(1e300)
    except Exception as e:                   # 40 iterations reached before tend, as configured
        assert "Maximum number of timesteps" in str(e)
    assert np.array_equal(bs.solution(k), ref.q)
    bs.close()


def test_batch_variants_agree():
    prob, insts = bench.batched_vc_config(n=5, seed=3, nmin=30, nmax=70)
    from pyclaw_b200.batch import BatchSolver
    results = []
    for v in range(_lib.load().claw2_batch_num_variants()):
        bs = BatchSolver(prob, insts)
        bs.init_controls([i["dt"] for i in insts], max_steps=10)
        bs.variant = v
        bs.advance(10)
        results.append([bs.solution(k) for k in range(len(insts))])
        bs.close()
    for r in results[1:]:
        for a, b in zip(results[0], r):
            assert np.array_equal(a, b)


def test_sharded_batch_shares_equal_the_whole_batch():
    """Each rank's share of a batch (pyclaw_b200.partition.ShardedBatch with
    the GPU BatchSolver), stepped here one share after the other on this GPU,
    gives every instance bit for bit the state of the unsharded batch."""
    from pyclaw_b200 import partition
    from pyclaw_b200.batch import BatchSolver
    prob, insts = bench.batched_vc_config(n=9, seed=11, nmin=20, nmax=120)
    dts = [i["dt"] for i in insts]
    whole = BatchSolver(prob, insts)
    whole.init_controls(dts, max_steps=25)
    whole.advance_graph(25, chunk=10)
    seen = set()
    for rank in range(3):
        sb = partition.ShardedBatch(prob, insts, rank, 3)
        sb.init_controls(dts, max_steps=25)
        sb.advance_graph(25, chunk=10)
        for k, q, ns, t in sb.local_results():
            seen.add(k)
            assert np.array_equal(q, whole.solution(k)), k
            assert ns == whole.controls()[k].numsteps and t == whole.controls()[k].t
        sb.close()
    assert seen == set(range(len(insts)))
    whole.close()


def test_batched_euler_one_state_tiles_equal_single_runs():
    """Euler instances with regions of one state run the batch's generic
    unsplit body; each must equal its solo run (the lean body, whose tiles of
    one state keep their cells) bit for bit."""
    rng = np.random.default_rng(4)
    insts = []
    for nx, ny in ((70, 45), (33, 90), (120, 64)):
        x = (np.arange(nx) + 0.5) / nx
        X = np.repeat(x[:, None], ny, axis=1)
        rho = np.where(X < 0.5, 1.0, 0.6)
        rho[:8, :8] += 0.2 * rng.random((8, 8))
        q = np.empty((4, nx, ny), order="F")
        q[0] = rho
        q[1] = rho * 0.2
        q[2] = 0.0
        q[3] = 1.0 / 0.4 + 0.5 * rho * 0.04
        insts.append(dict(q=q, aux=None, dx=1.0 / nx, dy=1.0 / ny, dt=0.2 / max(nx, ny)))
    prob = _abi.make_problem(rp=_abi.RP_EULER_4WAVE, num_eqn=4, num_waves=4, num_aux=0, mx=64, my=64, dx=1.0,
                             dy=1.0, order=2, transverse=2, mthlim=[4], params=(1.4, 0.4),
                             bc_lower=(_abi.BC_EXTRAP, _abi.BC_WALL), bc_upper=(_abi.BC_EXTRAP, _abi.BC_WALL))
    from pyclaw_b200.batch import BatchSolver
    bs = BatchSolver(prob, insts)
    bs.init_controls([i["dt"] for i in insts], max_steps=25)
    bs.advance(25)
    ctrls = bs.controls()
    for k in range(len(insts)):
        q_alone, c_alone = _alone(prob, insts[k], 25)
        assert ctrls[k].numsteps == c_alone.numsteps and ctrls[k].t == c_alone.t and ctrls[k].dt == c_alone.dt
        assert np.array_equal(bs.solution(k), q_alone)
    bs.close()


def test_tile_map_and_search_give_the_same_batch():
    """The one-CTA-per-tile variants read a tile's instance from the
    BatchSolver's tile -> instance map (claw2_batch_advance_map); without a
    map (claw2_batch_advance) they search the descriptors.  Both must give the
    same states, bit for bit."""
    prob, insts = bench.batched_vc_config(n=9, seed=11, nmin=40, nmax=130)
    from pyclaw_b200.batch import BatchSolver
    lib = _lib.load()
    nv = lib.claw2_batch_num_variants()
    per_tile = [v for v in range(nv) if v >= 10]
    assert per_tile
    for v in per_tile:
        sols = []
        for mapped in (True, False):
            bs = BatchSolver(prob, insts)
            bs.init_controls([i["dt"] for i in insts], max_steps=12)
            if mapped:
                bs.advance(12, v)
            else:
                desc, nt = bs._table(v)
                _lib.check(lib.claw2_batch_advance(ctypes.byref(bs.p), ctypes.c_void_p(desc.data_ptr()), bs.n, nt,
                                                   12, v, bs._stream()), "claw2_batch_advance")
            sols.append([bs.solution(k) for k in range(len(insts))])
            bs.close()
        for a, b in zip(*sols):
            assert np.array_equal(a, b)
