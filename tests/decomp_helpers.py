"""Test infrastructure for the domain decomposition (pyclaw_b200.decomp): a
CPU stand-in for decomp.Slab whose step is the oracle's, so that the
decomposition driver and its torch.distributed transport can run as gloo
ranks on CPU, and the rank worker used by tests/test_decomp_host.py."""
import ctypes
import os

import numpy as np


class OracleSlab(object):
    """decomp.Slab's interface on the host: the oracle steps the slab, the
    halo rows and the CFL scalar are CPU tensors."""

    def __init__(self, p, nranks, rank, q_global, aux_global, run):
        import torch
        from oracle import oracle as orc
        from pyclaw_b200 import decomp
        self.orc, self.lib = orc, orc.load()
        self.rank, self.nranks = rank, nranks
        self.p = decomp.slab_problem(p, nranks, rank)
        j0, j1 = decomp.slab_rows(p.my, nranks, rank)
        self.q = orc.new_qbc(self.p, q_global[:, :, j0:j1])
        orc.fill_ghosts(self.p, self.q, self.lib)
        self.aux = None
        if self.p.num_aux:
            mid, lo, hi = decomp.slab_aux(aux_global, p.my, nranks, rank)
            self.aux = orc.new_qbc(self.p, mid, self.p.num_aux)
            if lo is not None:
                self.aux[:, 2:-2, 0:2] = lo
            if hi is not None:
                self.aux[:, 2:-2, -2:] = hi
            orc.fill_aux_ghosts(self.p, self.aux, self.lib)
        self.ctrl = orc.control_init(0.0, run["dt_initial"], run["tend"], run["cfl_max"], run["cfl_desired"],
                                     lib=self.lib)
        n = self.p.num_eqn * 2 * (self.p.mx + 4)
        self.send = [torch.zeros(n, dtype=torch.float64), torch.zeros(n, dtype=torch.float64)]
        self.recv = [torch.zeros(n, dtype=torch.float64), torch.zeros(n, dtype=torch.float64)]
        self.cfl = torch.zeros(1, dtype=torch.float64)
        self.has = [rank > 0, rank < nranks - 1]
        self.qn = None

    def _rows(self, upper, ghost):
        my = self.p.my
        if ghost:
            return (my, my + 1) if upper else (-2, -1)
        return (my - 2, my - 1) if upper else (0, 1)

    def pack(self):
        for upper in (0, 1):
            if self.has[upper]:
                rows = [self.q[:, :, 2 + r] for r in self._rows(upper, False)]
                self.send[upper].copy_(self._t(np.stack(rows, axis=1).ravel()))

    def unpack(self):
        for upper in (0, 1):
            if self.has[upper]:
                b = self.recv[upper].numpy().reshape(self.p.num_eqn, 2, self.p.mx + 4)
                for k, r in enumerate(self._rows(upper, True)):
                    self.q[:, :, 2 + r] = b[:, k, :]

    def step(self):
        if self.ctrl.done:
            return
        self.qn = self.q.copy(order="F")
        cfl = self.orc.step_hyperbolic(self.p, self.qn, self.aux, self.ctrl.dt, self.lib)
        self.cfl[0] = cfl if np.isfinite(self.qn).all() else float("inf")

    def finish(self):
        if self.ctrl.done:
            return
        if self.lib.orc_control_update(ctypes.byref(self.ctrl), float(self.cfl[0])):
            self.q = self.qn
        self.orc.fill_ghosts(self.p, self.q, self.lib)

    def control(self):
        return self.ctrl

    def solution(self):
        return np.array(self.q[:, 2:-2, 2:-2])

    @staticmethod
    def _t(a):
        import torch
        return torch.from_numpy(np.ascontiguousarray(a))


def gloo_worker(rank, world, port, case, result_path):
    """One gloo rank: evolve its slab with the decomposition driver and the
    torch.distributed transport; rank 0 stores the gathered global solution."""
    import torch.distributed as dist
    from pyclaw_b200 import decomp
    p, q, aux, run = case()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        slab = OracleSlab(p, world, rank, q, aux, run)
        c = decomp.evolve([slab], decomp.DistTransport(slab), batch=4)
        parts = [None] * world
        dist.all_gather_object(parts, (slab.solution(), c.numsteps, c.t))
        if rank == 0:
            np.savez(result_path, q=np.concatenate([s for s, _, _ in parts], axis=2),
                     numsteps=np.array([n for _, n, _ in parts]), t=np.array([t for _, _, t in parts]))
    finally:
        dist.destroy_process_group()


def free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def euler_case():
    """A reduced shock-bubble (64 x 40 cells) run to t = 0.05."""
    import bench
    p, q, aux, run, tfinal = bench.shockbubble_config(64, 40)
    return p, q, aux, dict(run, tend=0.05)


def vc_case():
    """Variable-coefficient acoustics with layers across the cut (40 x 36)."""
    from pyclaw_b200 import _abi
    mx, my = 40, 36
    rng = np.random.default_rng(5)
    aux = np.empty((2, mx, my), order="F")
    aux[0] = 1.0 + 2.0 * (np.arange(my)[None, :] > my // 2 + 1) + 0.1 * rng.random((mx, my))
    aux[1] = 1.0 + 0.5 * rng.random((mx, my))
    x = (np.arange(mx) + 0.5) / mx
    y = (np.arange(my) + 0.5) / my
    X, Y = np.meshgrid(x, y, indexing="ij")
    q = np.zeros((3, mx, my), order="F")
    q[0] = np.exp(-((X - 0.4) ** 2 + (Y - 0.45) ** 2) / 0.02)
    p = _abi.make_problem(rp=_abi.RP_VC_ACOUSTICS, num_eqn=3, num_waves=2, num_aux=2, mx=mx, my=my, dx=1.0 / mx,
                          dy=1.0 / my, order=2, transverse=2, mthlim=[4],
                          bc_lower=(_abi.BC_WALL, _abi.BC_EXTRAP), bc_upper=(_abi.BC_EXTRAP, _abi.BC_WALL),
                          aux_bc_lower=(_abi.BC_EXTRAP, _abi.BC_EXTRAP),
                          aux_bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP))
    run = dict(cfl_max=1.0, cfl_desired=0.9, dt_initial=0.5 / mx, tend=0.3)
    return p, q, aux, run


def single_domain(p, q, aux, run):
    """The undecomposed run of the same problem through the oracle's controller."""
    from oracle import oracle as orc
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    abc = None
    if p.num_aux:
        abc = orc.new_qbc(p, aux, p.num_aux)
        orc.fill_aux_ghosts(p, abc)
    ctrl = orc.control_init(0.0, run["dt_initial"], run["tend"], run["cfl_max"], run["cfl_desired"])
    rc = orc.evolve(p, qbc, abc, ctrl)
    assert rc == 0, rc
    return np.array(qbc[:, 2:-2, 2:-2]), ctrl
