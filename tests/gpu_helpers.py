"""Helpers for the GPU parity tests: call libclaw2.so through its C ABI on
torch-held device buffers, converting to and from the reference layout."""
import ctypes

import numpy as np

from pyclaw_b200 import _abi, _lib


def torch():
    import torch as _t
    return _t


def to_dev(p, a, L):
    """reference-layout ghosted array (nc, mx+4, my+4) -> device-layout tensor"""
    t = torch()
    nc = a.shape[0]
    d = t.full((nc, L.rows, L.ld), float('nan'), dtype=t.float64)
    d[:, :, :p.mx + 4] = t.from_numpy(np.ascontiguousarray(a.transpose(0, 2, 1)))
    return d.reshape(-1).cuda()


def from_dev(p, d, nc, L):
    v = d.view(nc, L.rows, L.ld)[:, :, :p.mx + 4].permute(0, 2, 1).cpu().numpy()
    return np.asfortranarray(v)


def stream():
    return ctypes.c_void_p(torch().cuda.current_stream().cuda_stream)


def dev_step(p, qbc, auxbc, dt):
    """One claw2_step on copies of qbc/auxbc; returns (ghosted result, cfl)."""
    t = torch()
    lib = _lib.load()
    L = _lib.layout(p)
    qin = to_dev(p, qbc, L)
    qout = t.full_like(qin, float('nan'))
    aux = to_dev(p, auxbc, L) if auxbc is not None else t.zeros(1, dtype=t.float64, device='cuda')
    nscr = lib.claw2_scratch_bytes(ctypes.byref(p))
    scratch = t.zeros(nscr, dtype=t.uint8, device='cuda')
    cfl = t.zeros(1, dtype=t.float64, device='cuda')
    rc = lib.claw2_step(ctypes.byref(p), ctypes.c_void_p(qin.data_ptr()), ctypes.c_void_p(qout.data_ptr()),
                        ctypes.c_void_p(aux.data_ptr()), float(dt), ctypes.c_void_p(scratch.data_ptr()),
                        ctypes.c_void_p(cfl.data_ptr()), stream())
    _lib.check(rc, "claw2_step")
    t.cuda.synchronize()
    assert int(scratch[:4].view(t.int32).item()) == 0, "block-arrival counter not reset"
    return from_dev(p, qout, p.num_eqn, L), float(cfl.item())


def init_fields(p, seed=0):
    """Smooth-plus-noise physical initial data for any of the five solvers."""
    rng = np.random.default_rng(seed)
    mx, my = p.mx, p.my
    x = (np.arange(mx) + 0.5) / mx
    y = (np.arange(my) + 0.5) / my
    X, Y = np.meshgrid(x, y, indexing='ij')
    q = np.empty((p.num_eqn, mx, my), order='F')
    if p.rp in (_abi.RP_EULER_4WAVE, _abi.RP_EULER_5WAVE):
        rho = 1 + 0.5 * np.exp(-40 * ((X - .4) ** 2 + (Y - .5) ** 2)) + 0.1 * rng.random((mx, my))
        u = 0.8 * np.sin(2 * np.pi * Y) + 0.2 * rng.random((mx, my))
        v = 0.5 * np.cos(2 * np.pi * X)
        pr = 1 + 0.3 * rng.random((mx, my)) + 2 * (X < 0.3)
        q[0] = rho
        q[1] = rho * u
        q[2] = rho * v
        q[3] = pr / 0.4 + 0.5 * rho * (u * u + v * v)
        if p.num_eqn == 5:
            q[4] = (X > 0.5) * 1.0
    elif p.rp == _abi.RP_SHALLOW_ROE:
        h = 1 + (np.hypot(X - .5, Y - .5) < .2) + 0.1 * rng.random((mx, my))
        q[0] = h
        q[1] = h * (0.3 * rng.random((mx, my)) - 0.1)
        q[2] = h * 0.2 * np.sin(3 * X)
    else:
        q[0] = np.exp(-30 * ((X - .4) ** 2 + (Y - .6) ** 2)) + 0.1 * rng.random((mx, my))
        q[1] = 0.1 * rng.random((mx, my))
        q[2] = -0.05 * rng.random((mx, my))
    aux = None
    if p.num_aux:
        aux = np.empty((p.num_aux, mx, my), order='F')
        aux[0] = 1 + 3 * (X > 0.5)
        aux[1] = 1 + (Y > 0.3)
    return q, aux


SOLVERS = {
    "acoustics": dict(rp=_abi.RP_ACOUSTICS, num_eqn=3, num_waves=2, num_aux=0, params=(1.0, 4.0, 2.0, 2.0)),
    "vc_acoustics": dict(rp=_abi.RP_VC_ACOUSTICS, num_eqn=3, num_waves=2, num_aux=2, params=()),
    "euler4": dict(rp=_abi.RP_EULER_4WAVE, num_eqn=4, num_waves=4, num_aux=0, params=(1.4, 0.4)),
    "euler5": dict(rp=_abi.RP_EULER_5WAVE, num_eqn=5, num_waves=5, num_aux=0, params=(1.4, 0.4)),
    "shallow": dict(rp=_abi.RP_SHALLOW_ROE, num_eqn=3, num_waves=3, num_aux=0, params=(1.0,)),
}


def problem(name, mx, my, transverse, order=2, mthlim=(4,), bcl=(1, 1), bcu=(1, 1), abcl=(3, 3), abcu=(1, 1)):
    kw = dict(SOLVERS[name])
    return _abi.make_problem(mx=mx, my=my, dx=1.0 / mx, dy=1.0 / my, order=order, transverse=transverse,
                             mthlim=mthlim, bc_lower=bcl, bc_upper=bcu, aux_bc_lower=abcl,
                             aux_bc_upper=abcu, **kw)
