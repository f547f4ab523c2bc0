"""Batched form: many independent instances of one problem type, stepped together.

Every instance has its own grid size, spacing, aux fields and time-step
controller (its own dt from its own CFL number).  One launch of the batched
kernel takes one controlled step of every instance; the run of launches is
captured once into a CUDA graph and replayed.  The launch configuration
(threads per CTA, CTAs per SM of the persistent grid, and the tile edge, i.e.
the cells a CTA takes per work item) is chosen by `autotune`, which times the
candidates on the actual batch.

The reference steps one patch per call (ClawSolver2D.step_hyperbolic,
src/pyclaw/classic/solver.py:498-547); each instance here follows exactly that
step and Solver.evolve_to_time's controller (src/pyclaw/solver.py:632-691), so
an instance's result is bit-identical to running it alone.
"""
import ctypes
import json
import time

import numpy as np

from . import _abi, _lib


class BatchInstance(ctypes.Structure):
    """struct claw2_batch_instance (include/claw2.h)."""
    _fields_ = [
        ("q0", ctypes.c_void_p), ("q1", ctypes.c_void_p), ("aux", ctypes.c_void_p),
        ("ctrl", ctypes.c_void_p), ("partials", ctypes.c_void_p), ("ticket", ctypes.c_void_p),
        ("ld", ctypes.c_int64), ("plane", ctypes.c_int64),
        ("mx", ctypes.c_int32), ("my", ctypes.c_int32),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("nbx", ctypes.c_int32), ("nby", ctypes.c_int32),
        ("tile_begin", ctypes.c_int32), ("pad_", ctypes.c_int32),
    ]


def _lib_batch():
    return _lib.load()


class BatchSolver(object):
    """Advance many instances of one problem type together on one GPU.

    problem : a claw2 Problem holding the shared settings (Riemann solver,
              limiters, order, transverse mode, BCs, solver scalars); its
              grid fields are ignored.
    instances : list of dicts with keys q (num_eqn, mx, my), aux (num_aux, mx,
              my) or None, dx, dy, dt (initial dt).
    """

    def __init__(self, problem, instances, cfl_max=1.0, cfl_desired=0.9, dt_max=1e99, device=None):
        import torch
        if not torch.cuda.is_available():
            raise _lib.ClawLibraryError("pyclaw_b200 needs a CUDA device (sm_100a); none is available")
        self.torch = torch
        self.lib = _lib_batch()
        self.p = problem
        self.n = len(instances)
        self.device = torch.device(device if device is not None else "cuda")
        self.cfl_max, self.cfl_desired, self.dt_max = cfl_max, cfl_desired, dt_max
        meqn, maux = problem.num_eqn, problem.num_aux
        nv = self.lib.claw2_batch_num_variants()
        self.tile_of = {v: self.lib.claw2_batch_variant_tile(v) for v in range(nv)}
        edges = sorted(set(self.tile_of.values()), reverse=True)
        # one descriptor table per tile edge: the tiles of every instance
        # numbered consecutively; partials sized for the smallest edge
        tables = {e: (BatchInstance * self.n)() for e in edges}
        self.layouts = []
        self.problems = []
        offs_q, offs_a, offs_p = [], [], []
        nq = na = npart = 0
        ntiles = {e: 0 for e in edges}
        for k, inst in enumerate(instances):
            q = inst["q"]
            mx, my = q.shape[1], q.shape[2]
            pk = _abi.Problem.from_buffer_copy(problem)
            pk.mx, pk.my, pk.dx, pk.dy = mx, my, float(inst["dx"]), float(inst["dy"])
            _lib.check(self.lib.claw2_validate(ctypes.byref(pk)), "claw2_validate (instance %d)" % k)
            L = _lib.layout(pk)
            self.layouts.append(L)
            self.problems.append(pk)
            offs_q.append(nq)
            nq += 2 * L.q_elems
            offs_a.append(na)
            na += L.aux_elems
            offs_p.append(npart)
            most = 0
            for e in edges:
                nbx, nby = ctypes.c_int(), ctypes.c_int()
                _lib.check(self.lib.claw2_batch_tiles_for(e, mx, my, ctypes.byref(nbx), ctypes.byref(nby)),
                           "claw2_batch_tiles_for")
                d = tables[e][k]
                d.ld, d.plane, d.mx, d.my, d.dx, d.dy = L.ld, L.plane, mx, my, pk.dx, pk.dy
                d.nbx, d.nby, d.tile_begin = nbx.value, nby.value, ntiles[e]
                ntiles[e] += nbx.value * nby.value
                most = max(most, nbx.value * nby.value)
            npart += most
        self.ntiles_of = ntiles
        self.ntiles = ntiles[29]
        f64 = dict(dtype=torch.float64, device=self.device)
        self.qarena = torch.zeros(max(nq, 1), **f64)
        self.aarena = torch.zeros(max(na, 1), **f64)
        self.partials = torch.zeros(max(npart, 1), **f64)
        self.tickets = torch.zeros(self.n, dtype=torch.int32, device=self.device)
        csz = ctypes.sizeof(_abi.Control)
        self.ctrl = torch.zeros(self.n * csz, dtype=torch.uint8, device=self.device)
        self.ctrl_host = torch.zeros(self.n * csz, dtype=torch.uint8).pin_memory()
        base_q, base_a = self.qarena.data_ptr(), self.aarena.data_ptr()
        for descs in tables.values():
            for k in range(self.n):
                d, L = descs[k], self.layouts[k]
                d.q0 = base_q + 8 * offs_q[k]
                d.q1 = base_q + 8 * (offs_q[k] + L.q_elems)
                d.aux = (base_a + 8 * offs_a[k]) if maux > 0 else None
                d.ctrl = self.ctrl.data_ptr() + k * csz
                d.partials = self.partials.data_ptr() + 8 * offs_p[k]
                d.ticket = self.tickets.data_ptr() + 4 * k
        self.descs = tables[29]
        self.offs_q, self.offs_a = offs_q, offs_a
        self.desc_dev_of = {e: torch.frombuffer(bytearray(bytes(t)), dtype=torch.uint8).to(self.device)
                            for e, t in tables.items()}
        self.desc_dev = self.desc_dev_of[29]
        # tile -> instance maps, one per tile edge (the one-CTA-per-tile
        # variants read a tile's instance from it)
        self.map_dev_of = {}
        for e, t in tables.items():
            counts = [t[k].nbx * t[k].nby for k in range(self.n)]
            self.map_dev_of[e] = torch.from_numpy(
                np.repeat(np.arange(self.n, dtype=np.int32), counts)).to(self.device)
        self.variant = 0
        self._graphs = {}
        self.tuning = None
        for k, inst in enumerate(instances):
            self._upload(k, inst["q"], inst.get("aux"))
        self.init_controls([float(inst["dt"]) for inst in instances])

    # ---- buffers ---------------------------------------------------------------
    def _qview(self, k, which):
        L, meqn = self.layouts[k], self.p.num_eqn
        o = self.offs_q[k] + which * L.q_elems
        return self.qarena[o:o + L.q_elems].view(meqn, L.rows, L.ld)

    def _upload(self, k, q, aux):
        torch = self.torch
        pk, L = self.problems[k], self.layouts[k]
        g = _abi.NUM_GHOST
        v = self._qview(k, 0)
        v[:, g:g + pk.my, g:g + pk.mx].copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(q).transpose(0, 2, 1))))
        st = ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _lib.check(self.lib.claw2_fill_ghosts(ctypes.byref(pk), ctypes.c_void_p(v.data_ptr()), st), "fill_ghosts")
        if self.p.num_aux > 0:
            a = self.aarena[self.offs_a[k]:self.offs_a[k] + L.aux_elems].view(self.p.num_aux, L.rows, L.ld)
            a[:, g:g + pk.my, g:g + pk.mx].copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(aux).transpose(0, 2, 1))))
            _lib.check(self.lib.claw2_fill_aux_ghosts(ctypes.byref(pk), ctypes.c_void_p(a.data_ptr()), st),
                       "fill_aux_ghosts")

    def init_controls(self, dts, max_steps=1 << 40, tend=1e300):
        """Fresh controller per instance: evolve from t=0 towards tend with
        at most max_steps loop iterations (Solver.evolve_to_time semantics)."""
        csz = ctypes.sizeof(_abi.Control)
        base = self.ctrl_host.data_ptr()
        for k in range(self.n):
            c = _abi.Control.from_address(base + k * csz)
            _lib.check(self.lib.claw2_control_init(ctypes.byref(c), 0.0, float(dts[k]), float(tend), self.cfl_max,
                                                   self.cfl_desired, self.dt_max, 1, 0, int(max_steps),
                                                   self.cfl_desired), "claw2_control_init")
        self.ctrl.copy_(self.ctrl_host)

    def controls(self):
        self.ctrl_host.copy_(self.ctrl)
        self.torch.cuda.synchronize(self.device)
        csz = ctypes.sizeof(_abi.Control)
        base = self.ctrl_host.data_ptr()
        return [_abi.Control.from_buffer_copy(_abi.Control.from_address(base + k * csz)) for k in range(self.n)]

    def solution(self, k):
        """Instance k's current state (num_eqn, mx, my), Fortran order, on the host."""
        c = self.controls()[k]
        pk = self.problems[k]
        g = _abi.NUM_GHOST
        v = self._qview(k, c.cur)[:, g:g + pk.my, g:g + pk.mx].permute(0, 2, 1).cpu().numpy()
        return np.asfortranarray(v)

    # ---- stepping --------------------------------------------------------------
    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _table(self, v):
        """(device descriptor table, tile count) numbering the tiles of variant v's edge."""
        e = self.tile_of[v]
        return self.desc_dev_of[e], self.ntiles_of[e]

    def _map(self, v):
        """Device tile -> instance map of variant v's edge."""
        return ctypes.c_void_p(self.map_dev_of[self.tile_of[v]].data_ptr())

    def advance(self, nsteps, variant=None):
        """nsteps batched launches (no graph)."""
        v = self.variant if variant is None else variant
        desc, nt = self._table(v)
        _lib.check(self.lib.claw2_batch_advance_map(ctypes.byref(self.p), ctypes.c_void_p(desc.data_ptr()),
                                                    self.n, nt, self._map(v), int(nsteps), int(v), self._stream()),
                   "claw2_batch_advance_map")

    def advance_graph(self, nsteps, chunk=50):
        """nsteps launches replayed from CUDA graphs of `chunk` launches."""
        full, rest = divmod(int(nsteps), chunk)
        for count, reps in ((chunk, full), (rest, 1 if rest else 0)):
            if reps == 0:
                continue
            key = (count, self.variant)
            if key not in self._graphs:
                ge = ctypes.c_void_p()
                desc, nt = self._table(self.variant)
                _lib.check(self.lib.claw2_batch_graph_create_map(ctypes.byref(self.p),
                                                                 ctypes.c_void_p(desc.data_ptr()), self.n, nt,
                                                                 self._map(self.variant), count, self.variant,
                                                                 ctypes.byref(ge)),
                           "claw2_batch_graph_create_map")
                self._graphs[key] = ge
            for _ in range(reps):
                _lib.check(self.lib.claw2_graph_launch(self._graphs[key], self._stream()), "claw2_graph_launch")

    def autotune(self, steps=3, repeats=2):
        """Time every launch variant on this batch and keep the fastest.  The
        state and controllers are restored afterwards (all variants compute
        bit-identical results, so the choice affects speed only)."""
        torch = self.torch
        q_save = self.qarena.clone()
        c_save = self.ctrl.clone()
        nv = self.lib.claw2_batch_num_variants()
        times = {}
        for v in range(nv):
            try:
                self.advance(1, v)                   # configure + warm
            except _lib.ClawStatusError as e:
                if e.code == _abi.ERR_UNSUPPORTED:   # a launch shape this solver does not have
                    continue
                raise
            torch.cuda.synchronize(self.device)
            best = float("inf")
            for _ in range(repeats):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                self.advance(steps, v)
                e1.record()
                torch.cuda.synchronize(self.device)
                best = min(best, e0.elapsed_time(e1) / steps)
            th, cps = ctypes.c_int(), ctypes.c_int()
            self.lib.claw2_batch_variant_info(v, ctypes.byref(th), ctypes.byref(cps))
            times[v] = {"ms_per_launch": best, "threads": th.value, "ctas_per_sm": cps.value,
                        "tile": self.tile_of[v], "tiles": self._table(v)[1]}
        self.qarena.copy_(q_save)
        self.ctrl.copy_(c_save)
        self.tickets.zero_()
        torch.cuda.synchronize(self.device)
        self.variant = min(times, key=lambda v: times[v]["ms_per_launch"])
        self.desc_dev, self.ntiles = self._table(self.variant)
        self.tuning = {"chosen": self.variant, "candidates": times}
        return self.tuning

    def close(self):
        for ge in self._graphs.values():
            self.lib.claw2_graph_destroy(ge)
        self._graphs = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def describe(self):
        return json.dumps({"instances": self.n, "tiles": self.ntiles, "tuning": self.tuning})
