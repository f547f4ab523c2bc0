"""Sharding of the independent units (pyclaw_b200.partition) on CPU: the
split of batched instances and of adjoint shots, a batched run as 2 and 3
gloo ranks (the oracle stepping each rank's instances) equal to the same run
in one process, and the adjoint's partial gradients summed over 2 and 3 gloo
ranks equal to the whole-batch gradient."""
import numpy as np
import pytest
import torch.multiprocessing as mp

import decomp_helpers as D
import partition_helpers as PH
from pyclaw_b200 import partition


def test_partition_instances_covers_and_balances():
    rng = np.random.default_rng(0)
    sizes = [tuple(int(v) for v in rng.integers(64, 385, 2)) for _ in range(1024)]
    cost = [partition.tile_count(*s) for s in sizes]
    for n in (1, 2, 3, 4, 8):
        parts = partition.partition_instances(sizes, n)
        assert len(parts) == n
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(cost[k] for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(cost)
        assert parts == partition.partition_instances(sizes, n)     # deterministic
    assert partition.partition_instances([(10, 10)], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        partition.partition_instances(sizes, 0)


def test_shot_ranges():
    for S in (0, 1, 5, 64):
        for n in (1, 2, 3, 8):
            r = [partition.shot_range(S, n, k) for k in range(n)]
            assert r[0][0] == 0 and r[-1][1] == S
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            assert max(b - a for a, b in r) - min(b - a for a, b in r) <= 1
    with pytest.raises(ValueError):
        partition.shot_range(4, 2, 2)
    x = np.arange(10 * 7).reshape(10, 7)
    assert np.array_equal(partition.local_shots(x, 7, 1, 3, axis=1), x[:, 3:5])


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_equal_single_process_batch(tmp_path, world):
    nsteps = 12
    out = str(tmp_path / "batch.npz")
    mp.spawn(PH.batch_worker, args=(world, D.free_port(), nsteps, out), nprocs=world, join=True)
    r = np.load(out)
    prob, insts = PH.batch_case()
    ref = PH.OracleBatch(prob, insts)
    ref.init_controls([i["dt"] for i in insts], max_steps=nsteps)
    ref.advance_graph(nsteps)
    for k in range(len(insts)):
        assert np.array_equal(r["q%d" % k], ref.solution(k)), k
    assert list(r["steps"]) == [c.numsteps for c in ref.controls()]
    assert list(r["t"]) == [c.t for c in ref.controls()]
    assert min(r["steps"]) == nsteps


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_shot_gradients_sum_to_whole_batch(tmp_path, world):
    out = str(tmp_path / "shots.npz")
    mp.spawn(PH.shots_worker, args=(world, D.free_port(), out), nprocs=world, join=True)
    r = np.load(out)
    aux, q0, src, rec, wav, target = PH.shots_case()
    loss, grho, gc, gq = PH.shots_loss_and_grads(aux, q0, src, rec, wav, target)
    # the ranks add their shots' terms in another order: equal to round-off
    np.testing.assert_allclose(r["loss"], loss.numpy(), rtol=1e-13)
    for a, b in ((r["grho"], grho.numpy()), (r["gc"], gc.numpy())):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
    assert np.array_equal(r["gq"], gq.numpy())        # a shot's own gradient never mixes with others
