"""The multi-shot forward and the hand-written adjoint (include/claw2_adjoint.h)
against the plain FP64 torch transcription of the same step
(tests/torch_vc_step.py): traces bit for bit, gradients with respect to the
initial state and the per-cell material against torch.autograd, and central
finite differences on a 32x32 problem, at step sizes for which no limiter
branch changes between the two evaluations."""
import numpy as np
import pytest
import torch

import torch_vc_step as tv

pytestmark = pytest.mark.gpu


def _smooth(mx, my, seed, X, Y):
    g = np.random.default_rng(seed)
    f = np.zeros((mx, my))
    for _ in range(4):
        kx, ky = g.integers(1, 3, 2)
        ph = g.random(2) * 6.28
        f += g.standard_normal() * np.sin(np.pi * kx * X / 2 + ph[0]) * np.cos(np.pi * ky * Y / 2 + ph[1])
    return f


def make_case(mx, my, S, N, seed=0, bcl=(1, 1), bcu=(1, 3), abcl=None, abcu=None, limiters=(4, 4), trans=2,
              order=2, amp=1.0):
    rng = np.random.default_rng(seed)
    dx, dy = 2.0 / mx, 2.0 / my
    X, Y = np.meshgrid((np.arange(mx) + 0.5) * dx - 1, (np.arange(my) + 0.5) * dy - 1, indexing="ij")
    rho = 1.0 + 0.5 * np.exp(-((X - 0.2) ** 2 + (Y + 0.3) ** 2) / 0.3 ** 2) + 0.05 * rng.random((mx, my))
    K = 4.0 + 2.0 * np.exp(-((X + 0.3) ** 2 + (Y - 0.1) ** 2) / 0.3 ** 2) + 0.1 * rng.random((mx, my))
    p0 = amp * (0.2 * np.exp(-(X ** 2 + Y ** 2) / 0.2 ** 2) + 0.05 * _smooth(mx, my, seed + 11, X, Y))
    dt = 0.9 * min(dx, dy) / np.sqrt(K / rho).max()
    t = dt * (np.arange(N) + 1)
    f0 = 4.0
    w = (1 - 2 * (np.pi * f0 * (t - 0.3)) ** 2) * np.exp(-(np.pi * f0 * (t - 0.3)) ** 2)
    wav = amp * np.stack([w * (1.0 - 0.3 * s) for s in range(S)], axis=1)
    src = [(int(rng.integers(0, mx)), my - 1) for _ in range(S)]
    rec = [(i, my - 1) for i in range(1, mx, 3)] + [(mx // 2, my // 3)]
    abcl = tuple(bcl) if abcl is None else abcl
    abcu = tuple(bcu) if abcu is None else abcu
    return dict(mx=mx, my=my, S=S, N=N, dx=dx, dy=dy, dt=dt, rho=rho, K=K, p0=p0, wav=wav, src=src, rec=rec,
                bcl=tuple(bcl), bcu=tuple(bcu), abcl=tuple(abcl), abcu=tuple(abcu), limiters=tuple(limiters),
                trans=trans, order=order, dir=_smooth(mx, my, seed + 12, X, Y))


def runner_for(c, checkpoint=("uniform", 7)):
    from pyclaw_b200.adjoint import AcousticShots
    mx = c["mx"]
    return AcousticShots(c["mx"], c["my"], c["dx"], c["dy"], c["S"], [i + mx * j for i, j in c["src"]],
                         [i + mx * j for i, j in c["rec"]], c["wav"], c["dt"], bc_lower=c["bcl"], bc_upper=c["bcu"],
                         aux_bc_lower=c["abcl"], aux_bc_upper=c["abcu"], order=c["order"], transverse=c["trans"],
                         limiters=c["limiters"], checkpoint=checkpoint)


def q0_of(p0, S):
    z = torch.zeros_like(p0)
    return torch.stack([torch.stack([p0, z, z])] * S)


def torch_traces(c, rho, K, p0, aux=None):
    if aux is None:
        aux = torch.stack([rho, torch.sqrt(K / rho)])
    return tv.run_shots(q0_of(p0, c["S"]), aux, c["dt"], c["dx"], c["dy"], c["src"], c["rec"],
                        torch.tensor(c["wav"]), trans=c["trans"], mthlim=c["limiters"], bcl=c["bcl"], bcu=c["bcu"],
                        abcl=c["abcl"], abcu=c["abcu"], order=c["order"])


def cuda_traces(runner, rho, K, p0, S):
    from pyclaw_b200.adjoint import material_aux, shots_traces
    return shots_traces(q0_of(p0, S), material_aux(rho, K), runner)


CASES = {
    "mc_trans2_extrap_wall": dict(),
    "minmod_trans1_periodic_x": dict(bcl=(2, 3), bcu=(2, 3), abcl=(2, 1), abcu=(2, 1), limiters=(1, 1), trans=1),
    "superbee_trans0_walls": dict(bcl=(3, 3), bcu=(3, 3), abcl=(3, 3), abcu=(3, 3), limiters=(2, 2), trans=0),
    "vanleer_trans2_periodic_y": dict(bcl=(1, 2), bcu=(1, 2), abcl=(1, 2), abcu=(1, 2), limiters=(3, 3)),
    "unlimited_wave1": dict(limiters=(0, 4)),
    "order1_trans2": dict(order=1),
    # waves of about 1e-156: squared norms are subnormal (a reciprocal of such a
    # norm overflows); the linear term of the loss keeps the adjoint O(1)
    "subnormal_wave_norms": dict(amp=1e-155),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_forward_traces_bitwise(name):
    c = make_case(24, 20, 2, 25, seed=1, **CASES[name])
    rho, K, p0 = (torch.tensor(c[k]) for k in ("rho", "K", "p0"))
    from pyclaw_b200.adjoint import material_aux, shots_traces
    aux = material_aux(rho.cuda(), K.cuda())       # both sides use the same (device-rounded) c
    ref = torch_traces(c, rho, K, p0, aux.cpu())
    r = runner_for(c)
    got = shots_traces(q0_of(p0.cuda(), c["S"]), aux, r).cpu()
    assert got.shape == ref.shape
    assert torch.equal(got, ref), float((got - ref).abs().max())


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("name", sorted(CASES))
def test_gradient_matches_autograd(name):
    c = make_case(24, 20, 2, 25, seed=2, **CASES[name])
    rho, K, p0 = (torch.tensor(c[k]) for k in ("rho", "K", "p0"))
    with torch.no_grad():
        target = torch_traces(c, rho * 1.05, K, p0)
    # a linear term with O(1) weights keeps the adjoint O(1) whatever the amplitude
    wts = torch.tensor(np.random.default_rng(7).standard_normal(tuple(target.shape)))
    leaves = [x.clone().requires_grad_(True) for x in (rho, K, p0)]
    tr = torch_traces(c, *leaves)
    L = 0.5 * ((tr - target) ** 2).sum() + (wts * tr).sum()
    L.backward()
    r = runner_for(c)
    dl = [x.cuda().requires_grad_(True) for x in (rho, K, p0)]
    trc = cuda_traces(r, *dl, c["S"])
    Lc = 0.5 * ((trc - target.cuda()) ** 2).sum() + (wts.cuda() * trc).sum()
    Lc.backward()
    assert abs(Lc.item() - L.item()) <= 1e-12 * abs(L.item())
    for name_, ref, got in zip(("rho", "K", "p0"), leaves, dl):
        assert bool(torch.isfinite(got.grad).all()), name_
        err = _rel(got.grad.cpu(), ref.grad)
        assert err < 1e-10, (name_, err)


def _no_flips(c, args_p, args_m):
    logs = []
    for args in (args_p, args_m):
        tv.BRANCH_LOG = []
        with torch.no_grad():
            torch_traces(c, *[a.cpu() for a in args])
        logs.append(tv.BRANCH_LOG)
    tv.BRANCH_LOG = None
    return all(torch.equal(a, b) for a, b in zip(*logs))


def test_finite_differences_32x32():
    """Central differences of the misfit along smooth directions in rho, K and
    p0 agree with the adjoint gradient to 1e-6 relative, at a step for which
    the torch transcription takes the same limiter branches at both points."""
    c = make_case(32, 32, 2, 40, seed=4)
    rho, K, p0 = (torch.tensor(c[k]).cuda() for k in ("rho", "K", "p0"))
    r = runner_for(c, ("uniform", 10))
    with torch.no_grad():
        target = cuda_traces(r, rho * 1.05, K * 0.97, p0, c["S"]).clone()

    def misfit(*args):
        return 0.5 * ((cuda_traces(r, *args, c["S"]) - target) ** 2).sum()

    leaves = [x.clone().requires_grad_(True) for x in (rho, K, p0)]
    misfit(*leaves).backward()
    d = torch.tensor(c["dir"]).cuda()
    for which in range(3):
        an = float((leaves[which].grad * d).sum())
        base = [rho, K, p0]
        scale = float(base[which].abs().max())
        ok = False
        for rel_eps in (1e-6, 1e-7, 1e-8, 1e-9):
            eps = rel_eps * scale
            ap = list(base); ap[which] = base[which] + eps * d
            am = list(base); am[which] = base[which] - eps * d
            if not _no_flips(c, ap, am):
                continue
            with torch.no_grad():
                fd = float((misfit(*ap) - misfit(*am)) / (2 * eps))
            assert abs(fd - an) <= 1e-6 * abs(an), (which, rel_eps, fd, an)
            ok = True
            break
        assert ok, "no step free of limiter branch changes for parameter %d" % which


def test_schedules_give_identical_gradients():
    c = make_case(28, 22, 3, 37, seed=5)
    rho, K, p0 = (torch.tensor(c[k]).cuda() for k in ("rho", "K", "p0"))
    grads = []
    for ck in (("uniform", 37), ("uniform", 5), ("binomial", 3), ("binomial", 1), ("binomial", 0)):
        r = runner_for(c, ck)
        leaves = [x.clone().requires_grad_(True) for x in (rho, K, p0)]
        (cuda_traces(r, *leaves, c["S"]) ** 2).sum().backward()
        grads.append([x.grad.clone() for x in leaves])
    for g in grads[1:]:
        for a, b in zip(grads[0], g):
            assert torch.equal(a, b)


def test_multi_shot_equals_single_shots():
    """Shots are independent: the S-shot run equals S one-shot runs."""
    c = make_case(26, 21, 3, 15, seed=6)
    rho, K, p0 = (torch.tensor(c[k]).cuda() for k in ("rho", "K", "p0"))
    all_tr = cuda_traces(runner_for(c), rho, K, p0, 3).detach()
    for s in range(3):
        c1 = dict(c, S=1, src=[c["src"][s]], wav=c["wav"][:, s:s + 1])
        one = cuda_traces(runner_for(c1), rho, K, p0, 1).detach()
        assert torch.equal(one[:, 0], all_tr[:, s])
