"""Sharding of independent units across ranks (one process per GPU).

Two forms of this package advance units that never exchange data while they
step: the instances of a batched run (each with its own grid and its own
time-step controller) and the shots of the adjoint (wavefields sharing the
material but not their states).  They split across ranks with no per-step
collective:

- batched instances: `partition_instances` assigns whole instances to ranks,
  balancing the tiles each rank steps (every tile costs the same); each rank
  runs its own BatchSolver and `ShardedBatch.gather` collects the final
  states once at the end;
- adjoint shots: `shot_range` gives each rank a contiguous range of shots;
  the loss and the gradient with respect to the shared material are sums
  over shots, so `reduce_shared` adds the ranks' partial values once at the
  end (one all-reduce); gradients with respect to a shot's initial state stay
  on the rank that owns the shot.

PetClaw decomposes one grid across processes (src/petclaw/state.py,
src/petclaw/cfl.py); that case has a per-step exchange and lives in
pyclaw_b200.decomp.  The reference has no batched or adjoint form, so these
two have no counterpart there.
"""
import numpy as np

TILE = 29          # cells per side of one tile of the batched kernel


def tile_count(mx, my, tile=TILE):
    """Tiles of one instance: the unit of work of the batched kernel."""
    return ((int(mx) + tile - 1) // tile) * ((int(my) + tile - 1) // tile)


def partition_instances(sizes, nranks):
    """Split instances of sizes [(mx, my), ...] across nranks.

    Longest-processing-time rule: instances in decreasing tile count (ties by
    index) each go to the rank with the fewest tiles so far (ties to the lower
    rank).  Deterministic, so every rank computes the same split without
    communicating.  Returns one sorted list of instance indices per rank; a
    rank may get none when there are fewer instances than ranks.
    """
    nranks = int(nranks)
    if nranks < 1:
        raise ValueError("nranks must be at least 1")
    cost = [tile_count(mx, my) for mx, my in sizes]
    order = sorted(range(len(cost)), key=lambda k: (-cost[k], k))
    load = [0] * nranks
    parts = [[] for _ in range(nranks)]
    for k in order:
        r = min(range(nranks), key=lambda j: (load[j], j))
        parts[r].append(k)
        load[r] += cost[k]
    return [sorted(p) for p in parts]


def shot_range(nshots, nranks, rank):
    """Contiguous shots [s0, s1) of one rank; sizes differ by at most one."""
    nshots, nranks, rank = int(nshots), int(nranks), int(rank)
    if not 0 <= rank < nranks:
        raise ValueError("rank %d out of range for %d ranks" % (rank, nranks))
    base, extra = divmod(nshots, nranks)
    s0 = rank * base + min(rank, extra)
    return s0, s0 + base + (1 if rank < extra else 0)


def reduce_shared(tensors, group=None):
    """Sum the ranks' partial values in place (one all-reduce per tensor): the
    loss and the gradients with respect to quantities all shots share."""
    import torch.distributed as dist
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return tensors


class ShardedBatch(object):
    """One rank's share of a batched run.

    problem, instances : as for pyclaw_b200.batch.BatchSolver (all ranks pass
        the full list; each keeps its own share).
    rank, nranks : this process and the number of processes.
    solver_factory : builds the per-rank solver from (problem, instances,
        **kwargs); BatchSolver by default.
    """

    def __init__(self, problem, instances, rank, nranks, solver_factory=None, group=None, **kwargs):
        if solver_factory is None:
            from .batch import BatchSolver
            solver_factory = BatchSolver
        self.rank, self.nranks, self.group = int(rank), int(nranks), group
        self.n = len(instances)
        sizes = [(inst["q"].shape[1], inst["q"].shape[2]) for inst in instances]
        self.parts = partition_instances(sizes, nranks)
        self.mine = self.parts[self.rank]
        self.tiles = sum(tile_count(*sizes[k]) for k in self.mine)
        self.solver = solver_factory(problem, [instances[k] for k in self.mine], **kwargs) if self.mine else None

    def init_controls(self, dts, **kwargs):
        """dts: initial dt of every instance (global order)."""
        if self.solver is not None:
            self.solver.init_controls([dts[k] for k in self.mine], **kwargs)

    def advance_graph(self, nsteps, chunk=50):
        if self.solver is not None:
            self.solver.advance_graph(nsteps, chunk=chunk)

    def autotune(self, **kwargs):
        return self.solver.autotune(**kwargs) if self.solver is not None else None

    def local_results(self):
        """[(global index, state (num_eqn, mx, my), numsteps, t)] of this rank."""
        if self.solver is None:
            return []
        ctrls = self.solver.controls()
        return [(k, self.solver.solution(j), int(ctrls[j].numsteps), float(ctrls[j].t))
                for j, k in enumerate(self.mine)]

    def gather(self, dst=0):
        """Collect every instance's final state on rank dst (one collective at
        the end of the run).  Returns, on dst, lists (states, numsteps, t) in
        global instance order; None on the other ranks."""
        import torch.distributed as dist
        mine = self.local_results()
        if self.nranks == 1:
            allp = [mine]
        else:
            allp = [None] * self.nranks if self.rank == dst else None
            dist.gather_object(mine, allp, dst=dst, group=self.group)
        if self.rank != dst:
            return None
        states, steps, times = [None] * self.n, [0] * self.n, [0.0] * self.n
        for part in allp:
            for k, q, ns, t in part:
                states[k], steps[k], times[k] = q, ns, t
        if any(s is None for s in states):
            raise RuntimeError("gather: some instances were not stepped by any rank")
        return states, steps, times

    def close(self):
        if self.solver is not None and hasattr(self.solver, "close"):
            self.solver.close()


def local_shots(array, nshots, rank, nranks, axis=0):
    """This rank's slice of a per-shot array (sources, wavelets, initial states)."""
    s0, s1 = shot_range(nshots, nranks, rank)
    a = np.asarray(array) if not hasattr(array, "narrow") else array
    if hasattr(a, "narrow"):
        return a.narrow(axis, s0, s1 - s0)
    idx = [slice(None)] * a.ndim
    idx[axis] = slice(s0, s1)
    return a[tuple(idx)]
