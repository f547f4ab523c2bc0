"""Host-side checks of the adjoint machinery (no GPU): the checkpoint
schedules replay every state exactly once in reverse order, the torch
transcription of the multi-shot step equals the C oracle bit for bit, and its
autograd gradient agrees with central differences (so it can serve as the
reference gradient of the GPU adjoint)."""
import math

import numpy as np
import pytest
import torch

import torch_vc_step as tv
from pyclaw_b200 import _abi
from pyclaw_b200.adjoint import AcousticShots, binomial_split, ricker


class _Fake(object):
    """Stands in for the device calls: state -> 1.5 state + n + 1, recorded adjoints."""

    def __init__(self, N, checkpoint):
        self.r = object.__new__(AcousticShots)
        self.r.torch = torch
        self.r.nsteps = N
        self.r.checkpoint = checkpoint
        self.r.new_states = lambda n=1: torch.zeros((n, 1), dtype=torch.float64)
        self.r.step = self.step
        self.r._adj = self.adj
        self.nstep = 0
        self.calls = []

    def step(self, qin, qout, n, traces=None):
        qout.copy_(1.5 * qin + (n + 1))
        self.nstep += 1

    def adj(self, state, n, g):
        self.calls.append((n, float(state[0])))


def _true_states(N):
    s = [0.25]
    for n in range(N):
        s.append(1.5 * s[-1] + (n + 1))
    return s


@pytest.mark.parametrize("N,snaps", [(1, 0), (2, 0), (7, 0), (10, 1), (37, 2), (37, 3), (100, 4), (64, 6)])
def test_binomial_schedule_replays_states_in_reverse(N, snaps):
    f = _Fake(N, ("binomial", snaps))
    f.r._tmp = f.r.new_states(1)[0]
    slots = [f.r.new_states(1)[0] for _ in range(snaps)]
    q0 = torch.full((1,), 0.25, dtype=torch.float64)
    f.r._reverse_binomial(0, N, q0, slots, None)
    truth = _true_states(N)
    assert [c[0] for c in f.calls] == list(range(N - 1, -1, -1))
    for n, v in f.calls:
        assert v == truth[n]
    assert float(q0[0]) == 0.25                      # the initial state is kept intact
    if snaps >= 1:
        # forward recomputation of the binomial schedule: at most r*N steps with
        # r the smallest repetition count such that C(snaps + r, snaps) >= N
        r = 0
        while math.comb(snaps + r, snaps) < N:
            r += 1
        assert f.nstep <= max(r, 1) * N


@pytest.mark.parametrize("N,K", [(1, 5), (20, 20), (37, 5), (40, 20), (41, 7)])
def test_uniform_schedule_replays_states_in_reverse(N, K):
    f = _Fake(N, ("uniform", K))
    truth = _true_states(N)
    ckpt = {n: torch.tensor([truth[n]], dtype=torch.float64) for n in range(0, N, K)}
    f.r._reverse_uniform(K, ckpt, None)
    assert [c[0] for c in f.calls] == list(range(N - 1, -1, -1))
    for n, v in f.calls:
        assert v == truth[n]
    assert f.nstep == N - len(ckpt)                   # each segment recomputed once


def test_binomial_split_bounds():
    for snaps in range(1, 6):
        for n in range(2, 200):
            m = binomial_split(n, snaps)
            assert 1 <= m < n
            r = 0
            while math.comb(snaps + r, snaps) < n:
                r += 1
            assert n - m <= math.comb(snaps - 1 + r, snaps - 1)


def test_ricker_peak():
    assert ricker(0.3, 4.0, 0.3) == 1.0
    t = np.linspace(0, 0.6, 601)
    w = ricker(t, 4.0, 0.3)
    assert abs(w.sum() * 1e-3) < 1e-3                 # zero mean


def _case(mx=18, my=14, S=2, N=10, seed=0, bcl=(1, 1), bcu=(1, 3)):
    rng = np.random.default_rng(seed)
    aux = np.stack([1 + 3 * rng.random((mx, my)), 1 + rng.random((mx, my))])
    q0 = 0.1 * rng.standard_normal((S, 3, mx, my))
    src = [(int(rng.integers(0, mx)), my - 1) for _ in range(S)]
    rec = [(i, my - 1) for i in range(0, mx, 4)]
    wav = rng.standard_normal((N, S))
    return aux, q0, src, rec, wav


def test_transcription_matches_oracle_with_sources(orc):
    mx, my, N = 18, 14, 10
    for bcl, bcu, lim in (((1, 1), (1, 3), (4, 4)), ((2, 3), (2, 3), (1, 2))):
        aux, q0, src, rec, wav = _case(mx, my, 2, N, 3, bcl, bcu)
        abcl = [1 if b == 3 else b for b in bcl]
        abcu = [1 if b == 3 else b for b in bcu]
        dx, dy = 2.0 / mx, 2.0 / my
        dt = 0.4 * dx / 2
        tr = tv.run_shots(torch.tensor(q0), torch.tensor(aux), dt, dx, dy, src, rec, torch.tensor(wav), mthlim=lim,
                          bcl=bcl, bcu=bcu, abcl=abcl, abcu=abcu).numpy()
        p = _abi.make_problem(rp=_abi.RP_VC_ACOUSTICS, num_eqn=3, num_waves=2, num_aux=2, mx=mx, my=my, dx=dx,
                              dy=dy, order=2, transverse=2, mthlim=lim, bc_lower=bcl, bc_upper=bcu,
                              aux_bc_lower=abcl, aux_bc_upper=abcu)
        abc = orc.new_qbc(p, aux, 2)
        orc.fill_aux_ghosts(p, abc)
        for s in range(2):
            qbc = orc.new_qbc(p, q0[s])
            orc.fill_ghosts(p, qbc)
            for n in range(N):
                qnew = qbc.copy(order="F")
                orc.step2(p, qbc, qnew, abc, dt)
                qnew[0, 2 + src[s][0], 2 + src[s][1]] += wav[n, s]
                qbc = qnew
                orc.fill_ghosts(p, qbc)
                assert np.array_equal(tr[n, s], [qbc[0, 2 + i, 2 + j] for i, j in rec])


def test_transcription_gradient_matches_finite_differences():
    mx, my, S, N = 16, 14, 2, 16
    aux, q0, src, rec, wav = _case(mx, my, S, N, 5)
    dx, dy = 2.0 / mx, 2.0 / my
    dt = 0.4 * dx / 2
    rng = np.random.default_rng(9)
    target = torch.tensor(rng.standard_normal((N, S, len(rec)))) * 0.01
    rho = torch.tensor(aux[0], requires_grad=True)
    c = torch.tensor(aux[1], requires_grad=True)

    def loss(rho_, c_):
        tr = tv.run_shots(torch.tensor(q0), torch.stack([rho_, c_]), dt, dx, dy, src, rec, torch.tensor(wav),
                          bcl=(1, 1), bcu=(1, 3), abcl=(1, 1), abcu=(1, 1))
        return 0.5 * ((tr - target) ** 2).sum()

    loss(rho, c).backward()
    d = torch.tensor(rng.standard_normal((2, mx, my)))
    an = float((rho.grad * d[0]).sum() + (c.grad * d[1]).sum())
    eps = 1e-6
    with torch.no_grad():
        fd = float((loss(rho + eps * d[0], c + eps * d[1]) - loss(rho - eps * d[0], c - eps * d[1])) / (2 * eps))
    assert abs(fd - an) <= 1e-6 * abs(an)
