"""The branch-free division of the Riemann solvers and the limiter.

The kernels divide with FastDiv (pyclaw_b200/csrc/claw2_fastdiv.cuh): a
Newton-Raphson quotient plus a proof, from the exact FMA remainder, that the
quotient is the correctly rounded one; a solve whose proofs did not all pass
is redone with IEEE division.  These tests call the division on the GPU
through claw2_fastdiv_check and require, over many millions of operand pairs
(random over the whole exponent range, typical solver magnitudes and the hard
cases of division), that every quotient it marks as proven equals the IEEE
quotient bit for bit (numpy's division on the host), that the proof fails for
every operand outside its range, and that it passes for nearly all operands of
ordinary size.
"""
import ctypes

import numpy as np
import pytest

import gpu_helpers as H
from pyclaw_b200 import _lib

pytestmark = pytest.mark.gpu


def _fastdiv(a, b):
    t = H.torch()
    lib = _lib.load()
    da = t.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    db = t.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).cuda()
    q = t.empty_like(da)
    ok = t.empty(da.shape, dtype=t.uint8, device='cuda')
    rc = lib.claw2_fastdiv_check(ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(db.data_ptr()),
                                 ctypes.c_void_p(q.data_ptr()), ctypes.c_void_p(ok.data_ptr()), da.numel(),
                                 H.stream())
    assert rc == 0, _lib.load().claw2_strerror(rc)
    t.cuda.synchronize()
    return q.cpu().numpy(), ok.cpu().numpy().astype(bool)


def _bits(x):
    return np.ascontiguousarray(x).view(np.uint64)


def _check_proven(a, b):
    """Every proven quotient equals numpy's IEEE quotient bit for bit (NaN
    never proven).  Returns the proven fraction."""
    q, ok = _fastdiv(a, b)
    with np.errstate(all='ignore'):
        ref = a / b
    bad = ok & (_bits(q) != _bits(ref))
    assert not bad.any(), (a[bad][:5], b[bad][:5], q[bad][:5], ref[bad][:5])
    return ok.mean(), ok


def _random_doubles(rng, n, emin, emax):
    """Random signs, significands and exponents in [emin, emax]."""
    mant = rng.integers(0, 1 << 52, n, dtype=np.uint64)
    exp = rng.integers(emin + 1023, emax + 1023 + 1, n).astype(np.uint64)
    sign = rng.integers(0, 2, n, dtype=np.uint64) << np.uint64(63)
    return (sign | (exp << np.uint64(52)) | mant).view(np.float64)


def test_random_over_the_exponent_range():
    rng = np.random.default_rng(20261203)
    n = 1 << 23
    for _ in range(4):
        a = _random_doubles(rng, n, -1022, 1023)
        b = _random_doubles(rng, n, -1022, 1023)
        _check_proven(a, b)


def test_ordinary_magnitudes_are_nearly_always_proven():
    rng = np.random.default_rng(7)
    n = 1 << 23
    for scale in (1.0, 1e-6, 1e6):
        a = rng.standard_normal(n) * scale
        b = rng.uniform(0.01, 100.0, n) * rng.choice([-1.0, 1.0], n)
        frac, _ = _check_proven(a, b)
        assert frac > 1.0 - 1e-6, frac
        a = _random_doubles(rng, n, -200, 200)
        b = _random_doubles(rng, n, -200, 200)
        frac, _ = _check_proven(a, b)
        assert frac > 1.0 - 1e-6, frac


def test_hard_significands():
    """Divisors with significands all ones or near it and near 1.0, exact
    quotients (a = b*m), quotients that are powers of two, a == b."""
    rng = np.random.default_rng(11)
    n = 1 << 22
    ones = np.uint64((1 << 52) - 1)
    k = rng.integers(0, 64, n, dtype=np.uint64)
    # exponents within +-200, so that every quotient is inside the proof's range
    exp = rng.integers(1023 - 200, 1023 + 200, n).astype(np.uint64) << np.uint64(52)
    near_ones = (exp | (ones - k)).view(np.float64)
    near_one = (exp | k).view(np.float64)
    a = _random_doubles(rng, n, -200, 200)
    for b in (near_ones, near_one):
        frac, _ = _check_proven(a, b)
        assert frac > 1.0 - 1e-6
        # these quotients lie next to a power of two, where the proof uses the
        # smaller gap on both sides: correct, but a few per cent go to IEEE
        frac, _ = _check_proven(near_ones, b)
        assert frac > 0.9
        frac, _ = _check_proven(near_one, b)
        assert frac > 0.9
    # exact quotients: small integers times b, powers of two
    m = rng.integers(1, 1 << 20, n).astype(np.float64)
    b = _random_doubles(rng, n, -300, 300)
    frac, ok = _check_proven(m * b, b)
    assert frac > 1.0 - 1e-6
    p2 = np.ldexp(1.0, rng.integers(-200, 200, n))
    frac, _ = _check_proven(p2 * b, b)
    assert frac > 1.0 - 1e-6
    frac, _ = _check_proven(b, b)
    assert frac == 1.0


def test_zeros_signs_and_out_of_range_operands():
    tiny = np.nextafter(0.0, 1.0)
    big = np.finfo(np.float64).max
    specials = np.array([0.0, -0.0, 1.0, -1.0, 3.0, tiny, -tiny, 2.2250738585072014e-308, big, -big,
                         np.inf, -np.inf, np.nan, 2.0 ** -480, 2.0 ** -481, 2.0 ** 543, 2.0 ** 544,
                         1e-300, 1e300, 0.1, 7.0])
    a, b = np.meshgrid(specials, specials, indexing='ij')
    a, b = a.ravel(), b.ravel()
    q, ok = _fastdiv(a, b)
    with np.errstate(all='ignore'):
        ref = a / b
    assert not (ok & (_bits(q) != _bits(ref))).any()
    # zero dividends with ordinary divisors: proven, with the IEEE sign of zero
    for x in (0.0, -0.0):
        for y in (1.0, -1.0, 3.0, -7.0, 1e-100, 1e100):
            qq, oo = _fastdiv(np.array([x]), np.array([y]))
            assert oo[0] and _bits(qq)[0] == _bits(np.array([x / y]))[0], (x, y)
    # never proven: zero, subnormal, infinite, NaN or out-of-range divisors
    for y in (0.0, -0.0, tiny, np.inf, np.nan, 1e-300, 1e300, big):
        _, oo = _fastdiv(np.array([1.0, 0.0, -2.5]), np.full(3, y))
        assert not oo.any(), y
    # never proven: quotients out of range, infinite or NaN dividends
    _, oo = _fastdiv(np.array([1e-150, 1e150, np.inf, np.nan]), np.array([1e100, 1e-100, 1.0, 1.0]))
    assert not oo.any()
