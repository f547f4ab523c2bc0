"""Domain decomposition of one grid over several GPUs (one slab per process).

The reference parallelises a patch with PETSc (PetClaw): a distributed array
whose ghost rows are exchanged with the neighbours before every step
(DA.globalToLocal, src/petclaw/state.py:268) and a global max of the CFL
number (src/petclaw/cfl.py:30-31).  Here the grid is cut into slabs of rows
(the y direction), one per rank; a slab's sides that face another slab are
custom sides whose two ghost rows hold the neighbour's two boundary rows.
Every step runs, on every slab and asynchronously on its stream:

    halo pack -> exchange with the neighbours -> halo unpack -> step (local CFL)
    -> max of the CFL numbers over all slabs -> controller update -> ghost fill

so the step-size control stays on the device (the CFL max is a device
collective; every slab applies the same update and stays in step).  A cell's
update uses exactly the values the single-grid step uses, and a max is exact,
so the decomposed run equals the single-grid run bit for bit.

`Slab` wraps the device buffers and kernels of one slab.  Transports move the
halo buffers and reduce the CFL: `DistTransport` over torch.distributed (NCCL
between GPUs, gloo on CPU), `LocalTransport` for several slabs driven by one
process (used to check the decomposition on a single GPU: no kernel waits on
another, the exchange is a device copy).
"""
import ctypes

from . import _abi, _lib


def slab_rows(my, nranks, rank):
    """Rows [j0, j1) of the global grid that slab `rank` owns (as even as possible)."""
    base, extra = divmod(int(my), int(nranks))
    j0 = rank * base + min(rank, extra)
    return j0, j0 + base + (1 if rank < extra else 0)


def slab_problem(p, nranks, rank):
    """The claw2_problem of one slab: my of its rows, custom y sides (state
    and aux) where it faces another slab."""
    if nranks > 1 and (p.bc_lower[1] == _abi.BC_PERIODIC or p.aux_bc_lower[1] == _abi.BC_PERIODIC):
        raise NotImplementedError("periodic boundaries across the cut direction are not decomposed")
    q = _abi.Problem.from_buffer_copy(p)
    j0, j1 = slab_rows(p.my, nranks, rank)
    q.my = j1 - j0
    if rank > 0:
        q.bc_lower[1] = _abi.BC_CUSTOM
        q.aux_bc_lower[1] = _abi.BC_CUSTOM
    if rank < nranks - 1:
        q.bc_upper[1] = _abi.BC_CUSTOM
        q.aux_bc_upper[1] = _abi.BC_CUSTOM
    return q


def slab_aux(aux_global, my, nranks, rank):
    """The slab's aux (num_aux, mx, my_slab) and, where it has a neighbour,
    the two rows beyond each side that its ghost rows take from that
    neighbour (num_aux, mx, 2), or None."""
    j0, j1 = slab_rows(my, nranks, rank)
    lo = aux_global[:, :, j0 - 2:j0] if rank > 0 else None
    hi = aux_global[:, :, j1:j1 + 2] if rank < nranks - 1 else None
    return aux_global[:, :, j0:j1], lo, hi


class Slab(object):
    """Device state of one slab and the kernels of one decomposed step."""

    def __init__(self, p, nranks, rank, device=None):
        import torch
        from .device import DeviceState
        self.torch = torch
        self.rank, self.nranks = rank, nranks
        self.global_p = p
        self.p = slab_problem(p, nranks, rank)
        self.rows = slab_rows(p.my, nranks, rank)
        if self.p.my < 2:
            raise ValueError("a slab needs at least 2 rows")
        self.dev = DeviceState(self.p, device)
        self.lib = self.dev.lib
        n = self.p.num_eqn * 2 * (self.p.mx + 2 * _abi.NUM_GHOST)
        f64 = dict(dtype=torch.float64, device=self.dev.device)
        self.send = [torch.zeros(n, **f64), torch.zeros(n, **f64)]     # lower, upper
        self.recv = [torch.zeros(n, **f64), torch.zeros(n, **f64)]
        self.cfl = torch.zeros(1, **f64)
        self.has = [rank > 0, rank < nranks - 1]                       # neighbour below / above

    def upload(self, q_global, aux_global=None):
        """Set the slab from the global initial state (num_eqn, mx, my) and
        aux.  aux is constant: the ghost rows facing a neighbour get the
        neighbour's rows once, before the slab's own aux fill computes the
        ghost columns of every row, as the single-grid fill does."""
        import numpy as np
        j0, j1 = self.rows
        if aux_global is not None and self.p.num_aux > 0:
            mid, lo, hi = slab_aux(aux_global, self.global_p.my, self.nranks, self.rank)
            d, g = self.dev, _abi.NUM_GHOST
            d.upload_aux(mid)
            v = d.aux[:d.L.aux_elems].view(self.p.num_aux, d.L.rows, d.L.ld)
            for rows, at in ((lo, 0), (hi, self.p.my + g)):
                if rows is not None:
                    t = self.torch.from_numpy(np.ascontiguousarray(np.asarray(rows, dtype=np.float64)
                                                                   .transpose(0, 2, 1)))
                    v[:, at:at + g, g:g + self.p.mx].copy_(t)
            _lib.check(self.lib.claw2_fill_aux_ghosts(ctypes.byref(self.p), d.ptr(d.aux), d.stream),
                       "claw2_fill_aux_ghosts")
        self.dev.upload_q(q_global[:, :, j0:j1])

    def init_control(self, c):
        ctypes.memmove(self.dev.ctrl_host.data_ptr(), ctypes.addressof(c), ctypes.sizeof(c))
        self.dev.ctrl.copy_(self.dev.ctrl_host)

    def _a(self):
        d = self.dev
        return (ctypes.byref(self.p), d.ptr(d.q[0]), d.ptr(d.q[1]))

    def pack(self):
        d = self.dev
        for upper in (0, 1):
            if self.has[upper]:
                _lib.check(self.lib.claw2_halo_pack(*self._a(), d.ptr(d.ctrl), upper, d.ptr(self.send[upper]),
                                                    d.stream), "claw2_halo_pack")

    def unpack(self):
        d = self.dev
        for upper in (0, 1):
            if self.has[upper]:
                _lib.check(self.lib.claw2_halo_unpack(*self._a(), d.ptr(d.ctrl), upper, d.ptr(self.recv[upper]),
                                                      d.stream), "claw2_halo_unpack")

    def step(self):
        d = self.dev
        _lib.check(self.lib.claw2_step_ctrl(*self._a(), d.ptr(d.aux), d.ptr(d.ctrl), d.ptr(d.scratch),
                                            d.ptr(self.cfl), d.stream), "claw2_step_ctrl")

    def finish(self):
        d = self.dev
        _lib.check(self.lib.claw2_control_apply(d.ptr(d.ctrl), d.ptr(self.cfl), d.stream), "claw2_control_apply")
        _lib.check(self.lib.claw2_fill_ghosts_ctrl(*self._a(), d.ptr(d.ctrl), d.stream), "claw2_fill_ghosts_ctrl")

    def control(self):
        d = self.dev
        d.ctrl_host.copy_(d.ctrl)
        self.torch.cuda.synchronize(d.device)
        out = _abi.Control()
        ctypes.memmove(ctypes.addressof(out), d.ctrl_host.data_ptr(), ctypes.sizeof(out))
        return out

    def solution(self):
        """The slab's current interior (num_eqn, mx, my_slab) on the host."""
        self.dev.cur = self.control().cur
        return self.dev.download_q()


class LocalTransport(object):
    """Several slabs in one process: halo buffers are copied, the CFL max is
    taken over the slabs' device scalars (all on the current stream)."""

    def __init__(self, slabs):
        self.slabs = slabs

    def exchange(self):
        s = self.slabs
        for k in range(len(s) - 1):
            s[k + 1].recv[0].copy_(s[k].send[1])       # rows my-2, my-1 of k -> ghost rows -2, -1 of k+1
            s[k].recv[1].copy_(s[k + 1].send[0])       # rows 0, 1 of k+1 -> ghost rows my, my+1 of k

    def max_cfl(self):
        torch = self.slabs[0].torch
        m = torch.stack([s.cfl for s in self.slabs]).amax(dim=0)
        for s in self.slabs:
            s.cfl.copy_(m)


class DistTransport(object):
    """One slab per rank of a torch.distributed process group (NCCL between
    GPUs, gloo on CPU)."""

    def __init__(self, slab, group=None):
        import torch.distributed as dist
        self.dist, self.slab, self.group = dist, slab, group

    def exchange(self):
        dist, s = self.dist, self.slab
        ops = []
        if s.has[0]:
            ops.append(dist.P2POp(dist.isend, s.send[0], s.rank - 1, self.group))
            ops.append(dist.P2POp(dist.irecv, s.recv[0], s.rank - 1, self.group))
        if s.has[1]:
            ops.append(dist.P2POp(dist.isend, s.send[1], s.rank + 1, self.group))
            ops.append(dist.P2POp(dist.irecv, s.recv[1], s.rank + 1, self.group))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()

    def max_cfl(self):
        self.dist.all_reduce(self.slab.cfl, op=self.dist.ReduceOp.MAX, group=self.group)


def step_all(slabs, transport):
    """One decomposed step of every slab this process drives."""
    for s in slabs:
        s.pack()
    transport.exchange()
    for s in slabs:
        s.unpack()
        s.step()
    transport.max_cfl()
    for s in slabs:
        s.finish()


def evolve(slabs, transport, batch=8, max_iters=None):
    """Run decomposed steps until the (identical) controllers are done; the
    host looks at the controller once per batch of steps.  Returns the final
    claw2_control of the first slab."""
    it = 0
    while True:
        for _ in range(batch):
            step_all(slabs, transport)
        it += batch
        c = slabs[0].control()
        if c.done or (max_iters is not None and it >= max_iters):
            return c
