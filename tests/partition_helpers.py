"""Test infrastructure for pyclaw_b200.partition: a CPU stand-in for
BatchSolver whose instances the oracle steps, the gloo rank workers of
tests/test_partition_host.py and a small batch of uneven instances."""
import numpy as np


class OracleBatch(object):
    """BatchSolver's interface (init_controls, advance_graph, controls,
    solution) on the host: each instance is a ghosted array stepped by the
    oracle's evolve_to_time replay, one controlled step per launch."""

    def __init__(self, problem, instances, cfl_max=1.0, cfl_desired=0.9):
        from oracle import oracle as orc
        from pyclaw_b200 import _abi
        self.orc, self.lib = orc, orc.load()
        self.cfl_max, self.cfl_desired = cfl_max, cfl_desired
        self.problems, self.q, self.aux, self.ctrl = [], [], [], []
        for inst in instances:
            pk = _abi.Problem.from_buffer_copy(problem)
            pk.mx, pk.my = inst["q"].shape[1], inst["q"].shape[2]
            pk.dx, pk.dy = float(inst["dx"]), float(inst["dy"])
            qbc = orc.new_qbc(pk, inst["q"])
            orc.fill_ghosts(pk, qbc, self.lib)
            abc = None
            if pk.num_aux:
                abc = orc.new_qbc(pk, inst["aux"], pk.num_aux)
                orc.fill_aux_ghosts(pk, abc, self.lib)
            self.problems.append(pk)
            self.q.append(qbc)
            self.aux.append(abc)

    def init_controls(self, dts, max_steps=1 << 40, tend=1e300):
        self.ctrl = [self.orc.control_init(0.0, float(dt), tend, self.cfl_max, self.cfl_desired,
                                           max_steps=max_steps, lib=self.lib) for dt in dts]

    def advance_graph(self, nsteps, chunk=50):
        for _ in range(int(nsteps)):
            for pk, qbc, abc, c in zip(self.problems, self.q, self.aux, self.ctrl):
                if c.done:
                    continue
                limit = c.max_steps               # one controlled step per launch
                c.max_steps = c.iter + 1
                rc = self.orc.evolve(pk, qbc, abc, c, lib=self.lib)
                assert rc in (0, 5), rc
                c.max_steps = limit
                if c.iter < limit:
                    c.done, c.error = 0, 0

    def controls(self):
        return self.ctrl

    def solution(self, k):
        return np.array(self.q[k][:, 2:-2, 2:-2])


def batch_case(n=7, seed=3):
    """n small uneven vc-acoustics instances (the batched workload's setup)."""
    import bench
    prob, insts = bench.batched_vc_config(n=n, seed=seed, nmin=12, nmax=70)
    return prob, insts


def batch_worker(rank, world, port, nsteps, result_path):
    """One gloo rank: step its share of the batch with the oracle stand-in and
    gather every instance's state on rank 0."""
    import torch.distributed as dist
    from pyclaw_b200 import partition
    prob, insts = batch_case()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        sb = partition.ShardedBatch(prob, insts, rank, world, solver_factory=OracleBatch)
        sb.init_controls([i["dt"] for i in insts], max_steps=nsteps)
        sb.advance_graph(nsteps)
        out = sb.gather(dst=0)
        if rank == 0:
            states, steps, times = out
            np.savez(result_path, steps=np.array(steps), t=np.array(times),
                     **{"q%d" % k: s for k, s in enumerate(states)})
    finally:
        dist.destroy_process_group()


def shots_case(S=5, N=6, mx=14, my=12, seed=4):
    rng = np.random.default_rng(seed)
    aux = np.stack([1 + 3 * rng.random((mx, my)), 1 + rng.random((mx, my))])
    q0 = 0.1 * rng.standard_normal((S, 3, mx, my))
    src = [(int(rng.integers(0, mx)), my - 1) for _ in range(S)]
    rec = [(i, my - 1) for i in range(0, mx, 3)]
    wav = rng.standard_normal((N, S))
    target = 0.01 * rng.standard_normal((N, S, len(rec)))
    return aux, q0, src, rec, wav, target


def shots_loss_and_grads(aux, q0, src, rec, wav, target):
    """Misfit of the given shots and its gradients (rho, c, q0) through the
    plain-torch transcription of the step (autograd)."""
    import torch
    import torch_vc_step as tv
    mx, my = aux.shape[1], aux.shape[2]
    dx, dy = 2.0 / mx, 2.0 / my
    dt = 0.4 * dx / 2
    rho = torch.tensor(aux[0], requires_grad=True)
    c = torch.tensor(aux[1], requires_grad=True)
    q = torch.tensor(q0, requires_grad=True)
    tr = tv.run_shots(q, torch.stack([rho, c]), dt, dx, dy, src, rec, torch.tensor(wav),
                      bcl=(1, 1), bcu=(1, 3), abcl=(1, 1), abcu=(1, 1))
    loss = 0.5 * ((tr - torch.tensor(target)) ** 2).sum()
    loss.backward()
    return loss.detach().reshape(1), rho.grad, c.grad, q.grad


def shots_worker(rank, world, port, result_path):
    """One gloo rank: the misfit and gradients of its shots, then one sum
    all-reduce of the loss and the material gradients."""
    import torch.distributed as dist
    from pyclaw_b200 import partition
    aux, q0, src, rec, wav, target = shots_case()
    S = q0.shape[0]
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        s0, s1 = partition.shot_range(S, world, rank)
        loss, grho, gc, gq = shots_loss_and_grads(aux, partition.local_shots(q0, S, rank, world), src[s0:s1], rec,
                                                  partition.local_shots(wav, S, rank, world, axis=1),
                                                  partition.local_shots(target, S, rank, world, axis=1))
        partition.reduce_shared([loss, grho, gc])
        parts = [None] * world if rank == 0 else None
        dist.gather_object((s0, s1, gq.numpy()), parts, dst=0)
        if rank == 0:
            gq_all = np.zeros_like(q0)
            for a, b, g in parts:
                gq_all[a:b] = g
            np.savez(result_path, loss=loss.numpy(), grho=grho.numpy(), gc=gc.numpy(), gq=gq_all)
    finally:
        dist.destroy_process_group()
