"""Differentiable multi-shot variable-coefficient acoustics.

S wavefields ("shots") of 2D variable-coefficient acoustics, q = (p, u, v),
share one material, aux = (rho, c), and one fixed dt.  Every step is the
classic unsplit step (ClawSolver2D.step_hyperbolic with the vc_acoustics
Riemann solvers, src/pyclaw/classic/solver.py:498-547) run by the sm_100a
library, followed by a point source per shot (the wavelet sample of that
step added to the pressure of the source cell) and the pressure sampled at
the receiver cells.

`ShotsFunction` is a torch.autograd.Function from (q0, aux) to the receiver
traces.  Its backward runs the hand-written adjoint kernels (the transpose of
each step with the limiter branches frozen at the forward state) backwards in
time over states recomputed from checkpoints:

* ``checkpoint=("uniform", K)``: the forward keeps every K-th state; the
  backward recomputes one K-step segment at a time into a segment buffer.
* ``checkpoint=("binomial", s)``: s snapshot slots besides the initial state,
  placed by the binomial (revolve) rule of Griewank & Walther (ACM TOMS 26,
  2000), for runs whose states do not fit in memory.

Both schedules give bit-identical gradients (recomputation is
deterministic).  dt is a constant of the run, not differentiated.  The
reference has no adjoint; the forward step is the reference's.
"""
import ctypes
import math

import numpy as np

from . import _abi, _lib


def ricker(t, f0, t0):
    """Ricker wavelet (1 - 2 (pi f0 (t-t0))^2) exp(-(pi f0 (t-t0))^2)."""
    a = (np.pi * f0 * (np.asarray(t, dtype=np.float64) - t0)) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


def binomial_split(n, snaps):
    """Steps to advance before placing the next snapshot when n steps must be
    reversed with `snaps` free snapshot slots: with r the smallest number of
    repetitions such that C(snaps + r, snaps) >= n, the right part gets at most
    C(snaps - 1 + r, snaps - 1) steps (Griewank's binomial recursion
    beta(s, r) = beta(s-1, r) + beta(s, r-1))."""
    if n <= 1 or snaps <= 0:
        return 1
    r = 0
    while math.comb(snaps + r, snaps) < n:
        r += 1
    right = math.comb(snaps - 1 + r, snaps - 1)
    return max(1, n - right)


class AcousticShots(object):
    """Device buffers and schedules for one configuration of shots.

    mx, my, dx, dy : grid; nshots : S; src_cells : (S,) flat interior index
    i + mx*j of each shot's source (-1: none); rec_cells : (R,) flat indices
    of the receivers; wavelet : (N, S) or (N,) amplitude added at the source
    after step n; bc_lower/bc_upper, aux_bc_lower/aux_bc_upper : pyclaw BC
    codes (extrap 1, periodic 2, wall 3); order, transverse, limiters : as
    ClawSolver2D.
    """

    def __init__(self, mx, my, dx, dy, nshots, src_cells, rec_cells, wavelet, dt, *,
                 bc_lower=(1, 1), bc_upper=(1, 1), aux_bc_lower=None, aux_bc_upper=None,
                 order=2, transverse=2, limiters=(4, 4), checkpoint=("uniform", 20), device="cuda"):
        import torch
        if not torch.cuda.is_available():
            raise _lib.ClawLibraryError("pyclaw_b200 needs a CUDA device (sm_100a); none is available")
        self.torch = torch
        self.lib = _lib.load()
        self.device = torch.device(device)
        aux_bc_lower = tuple(bc_lower) if aux_bc_lower is None else aux_bc_lower
        aux_bc_upper = tuple(bc_upper) if aux_bc_upper is None else aux_bc_upper
        self.p = _abi.make_problem(rp=_abi.RP_VC_ACOUSTICS, num_eqn=3, num_waves=2, num_aux=2, mx=mx, my=my,
                                   dx=dx, dy=dy, order=order, transverse=transverse, mthlim=tuple(limiters),
                                   bc_lower=bc_lower, bc_upper=bc_upper, aux_bc_lower=aux_bc_lower,
                                   aux_bc_upper=aux_bc_upper)
        _lib.check(self.lib.claw2_validate(ctypes.byref(self.p)), "claw2_validate")
        self.L = _lib.layout(self.p)
        self.mx, self.my, self.S = mx, my, int(nshots)
        self.dt = float(dt)
        w = np.asarray(wavelet, dtype=np.float64)
        if w.ndim == 1:
            w = np.repeat(w[:, None], self.S, axis=1)
        self.nsteps = w.shape[0]
        self.checkpoint = tuple(checkpoint)
        f64 = dict(dtype=torch.float64, device=self.device)
        i32 = dict(dtype=torch.int32, device=self.device)
        self.wavelet = torch.tensor(w, **f64).contiguous()
        self.src = torch.tensor(np.asarray(src_cells, dtype=np.int32), **i32)
        self.rec = torch.tensor(np.asarray(rec_cells, dtype=np.int32), **i32)
        self.R = int(self.rec.numel())
        self.qe = int(self.L.q_elems)
        self.aux = torch.zeros(int(self.L.aux_elems), **f64)
        self.cfl = torch.zeros(self.S, **f64)
        nb = self.lib.claw2_shots_scratch_bytes(ctypes.byref(self.p), self.S)
        self.scratch = torch.zeros((nb + 7) // 8, **f64)
        self.cfl_max_seen = 0.0

    # ---- small helpers --------------------------------------------------------
    def _st(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def new_states(self, n=1):
        return self.torch.zeros((n, self.S * self.qe), dtype=self.torch.float64, device=self.device)

    def _interior(self, flat, ncomp):
        L, g = self.L, _abi.NUM_GHOST
        v = flat.view(self.S, ncomp, L.rows, L.ld)
        return v[:, :, g:g + self.my, g:g + self.mx]

    def set_aux(self, aux):
        """aux: (2, mx, my) tensor (rho, c); fills the ghost cells."""
        L, g = self.L, _abi.NUM_GHOST
        v = self.aux.view(2, L.rows, L.ld)
        v[:, g:g + self.my, g:g + self.mx].copy_(aux.detach().to(self.device, self.torch.float64).transpose(1, 2))
        _lib.check(self.lib.claw2_fill_aux_ghosts(ctypes.byref(self.p), ctypes.c_void_p(self.aux.data_ptr()),
                                                  self._st()), "claw2_fill_aux_ghosts")

    def set_state(self, buf, q0):
        """q0: (S, 3, mx, my) -> buf (ghosts filled)."""
        self._interior(buf, 3).copy_(q0.detach().to(self.device, self.torch.float64).transpose(2, 3))
        st = self._st()
        for s in range(self.S):
            _lib.check(self.lib.claw2_fill_ghosts(ctypes.byref(self.p), ctypes.c_void_p(buf.data_ptr() + 8 * s * self.qe),
                                                  st), "claw2_fill_ghosts")

    def step(self, qin, qout, n, traces=None):
        """q^{n+1} = step(q^n) + source; traces[n] recorded when given."""
        st = self._st()
        _lib.check(self.lib.claw2_shots_step(ctypes.byref(self.p), self.S, self.qe, ctypes.c_void_p(qin.data_ptr()),
                                             ctypes.c_void_p(qout.data_ptr()), ctypes.c_void_p(self.aux.data_ptr()),
                                             self.dt, ctypes.c_void_p(self.scratch.data_ptr()),
                                             ctypes.c_void_p(self.cfl.data_ptr()), st), "claw2_shots_step")
        amp = ctypes.c_void_p(self.wavelet[n].data_ptr())
        tr = ctypes.c_void_p(traces[n].data_ptr()) if traces is not None else None
        _lib.check(self.lib.claw2_shots_inject_record(ctypes.byref(self.p), self.S, self.qe,
                                                      ctypes.c_void_p(qout.data_ptr()),
                                                      ctypes.c_void_p(self.src.data_ptr()), amp, self.R,
                                                      ctypes.c_void_p(self.rec.data_ptr()), tr, st),
                   "claw2_shots_inject_record")

    def advance(self, buf, tmp, n0, n1):
        """buf holds q^{n0}; on return it holds q^{n1} (tmp is scratch)."""
        a, b = buf, tmp
        for n in range(n0, n1):
            self.step(a, b, n)
            a, b = b, a
        if a is not buf:
            buf.copy_(a)

    # ---- forward -----------------------------------------------------------------
    def forward(self, q0, aux):
        """Run all steps.  Returns traces (N, S, R) and the tape (aux and the
        checkpointed states) that `backward` needs."""
        torch = self.torch
        self.set_aux(aux)
        N = self.nsteps
        traces = torch.zeros((N, self.S, max(self.R, 1)), dtype=torch.float64, device=self.device)
        kind, arg = self.checkpoint
        cur, nxt = self.new_states(1)[0], self.new_states(1)[0]
        self.set_state(cur, q0)
        tape = {"aux": self.aux.clone(), "ckpt": {0: cur.clone()}}
        if kind == "uniform":
            K = int(arg)
            for n in range(N):
                self.step(cur, nxt, n, traces)
                cur, nxt = nxt, cur
                if (n + 1) % K == 0 and n + 1 < N:
                    tape["ckpt"][n + 1] = cur.clone()
        elif kind == "binomial":
            for n in range(N):
                self.step(cur, nxt, n, traces)
                cur, nxt = nxt, cur
        else:
            raise ValueError("checkpoint must be ('uniform', K) or ('binomial', snaps)")
        self.cfl_max_seen = float(self.cfl.max())
        return traces[:, :, :self.R], tape

    # ---- backward ------------------------------------------------------------------
    def _adjoint_step(self, state, n, lam_in, lam_out, gtraces):
        """lam_out = adjoint of step n+1 (from state q^n) applied to lam_in, folded,
        plus the trace gradient of q^n (recorded after step n)."""
        st = self._st()
        _lib.check(self.lib.claw2_shots_adjoint_step(ctypes.byref(self.p), self.S, self.qe,
                                                     ctypes.c_void_p(state.data_ptr()),
                                                     ctypes.c_void_p(self.aux.data_ptr()), self.dt,
                                                     ctypes.c_void_p(lam_in.data_ptr()),
                                                     ctypes.c_void_p(lam_out.data_ptr()),
                                                     ctypes.c_void_p(self.gaux.data_ptr()), 2 * self.L.plane, st),
                   "claw2_shots_adjoint_step")
        self._fold(lam_out, gtraces[n - 1] if n >= 1 else None)

    def _fold(self, lam, g):
        _lib.check(self.lib.claw2_shots_adjoint_fold(ctypes.byref(self.p), self.S, self.qe,
                                                     ctypes.c_void_p(lam.data_ptr()), self.R if g is not None else 0,
                                                     ctypes.c_void_p(self.rec.data_ptr()),
                                                     ctypes.c_void_p(g.data_ptr()) if g is not None else None,
                                                     self._st()), "claw2_shots_adjoint_fold")

    def backward(self, gtraces, tape):
        """gtraces (N, S, R): dLoss/dtraces of the forward that made `tape`.
        Returns (dL/dq0 (S,3,mx,my), dL/daux (2,mx,my))."""
        torch = self.torch
        N = self.nsteps
        self.aux.copy_(tape["aux"])
        g = torch.zeros((N, self.S, max(self.R, 1)), dtype=torch.float64, device=self.device)
        g[:, :, :self.R] = gtraces.to(self.device, torch.float64)
        self.gaux = torch.zeros(self.S * 2 * self.L.plane, dtype=torch.float64, device=self.device)
        lam = self.new_states(2)
        self._lam = [lam[0], lam[1]]
        self._fold(self._lam[0], g[N - 1])            # lambda^N: the last trace's gradient
        self._which = 0
        kind, arg = self.checkpoint
        if kind == "uniform":
            self._reverse_uniform(int(arg), tape["ckpt"], g)
        else:
            self._tmp = self.new_states(1)[0]
            slots = [self.new_states(1)[0] for _ in range(int(arg))]
            self._reverse_binomial(0, N, tape["ckpt"][0], slots, g)
        lam_fin = self._lam[self._which]
        _lib.check(self.lib.claw2_shots_fold_aux(ctypes.byref(self.p), self.S, 2 * self.L.plane,
                                                 ctypes.c_void_p(self.gaux.data_ptr()), self._st()),
                   "claw2_shots_fold_aux")
        gq0 = self._interior(lam_fin, 3).transpose(2, 3).clone()
        L, gh = self.L, _abi.NUM_GHOST
        ga = self.gaux.view(self.S, 2, L.rows, L.ld)[:, :, gh:gh + self.my, gh:gh + self.mx]
        gaux = ga.sum(dim=0).transpose(1, 2).contiguous()
        self._lam = self._tmp = self._w = None
        self.gaux = None
        return gq0, gaux

    def _adj(self, state, n, g):
        """One adjoint step from lambda^{n+1} to lambda^n using q^n."""
        a = self._lam[self._which]
        b = self._lam[1 - self._which]
        self._adjoint_step(state, n, a, b, g)
        self._which = 1 - self._which

    def _reverse_uniform(self, K, ckpt, g):
        N = self.nsteps
        seg = self.new_states(K)
        for s0 in sorted(ckpt, reverse=True):
            s1 = min(s0 + K, N)
            seg[0].copy_(ckpt[s0])
            for n in range(s0, s1 - 1):                # states q^{s0+1} .. q^{s1-1}
                self.step(seg[n - s0], seg[n - s0 + 1], n)
            for n in range(s1 - 1, s0 - 1, -1):
                self._adj(seg[n - s0], n, g)

    def _reverse_binomial(self, a, b, state_a, free, g):
        """Adjoint of steps a+1..b given q^a (kept intact) and free snapshot slots."""
        n = b - a
        if n == 1:
            self._adj(state_a, a, g)
            return
        if not free:
            for t in range(b - 1, a - 1, -1):
                self._tmp.copy_(state_a)
                w = self._scratch_state()
                self.advance(self._tmp, w, a, t)
                self._adj(self._tmp, t, g)
            return
        m = a + binomial_split(n, len(free))
        slot = free[0]
        slot.copy_(state_a)
        self.advance(slot, self._scratch_state(), a, m)
        self._reverse_binomial(m, b, slot, free[1:], g)
        self._reverse_binomial(a, m, state_a, free, g)

    def _scratch_state(self):
        if getattr(self, "_w", None) is None:
            self._w = self.new_states(1)[0]
        return self._w

def _function():
    import torch

    class ShotsFunction(torch.autograd.Function):
        """(q0 (S,3,mx,my), aux (2,mx,my)) -> traces (N,S,R), with the
        hand-written adjoint as backward."""

        @staticmethod
        def forward(ctx, q0, aux, runner):
            traces, tape = runner.forward(q0, aux)
            ctx.runner, ctx.tape = runner, tape
            return traces

        @staticmethod
        def backward(ctx, gtr):
            gq0, gaux = ctx.runner.backward(gtr.contiguous(), ctx.tape)
            ctx.tape = None
            return gq0, gaux, None

    return ShotsFunction


_FN = None


def shots_traces(q0, aux, runner):
    """Differentiable traces of the shots; aux = (rho, c) per cell."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(q0, aux, runner)


def material_aux(rho, K):
    """aux = (rho, c) with c = sqrt(K / rho), differentiable in (rho, K)."""
    import torch
    return torch.stack([rho, torch.sqrt(K / rho)])
