"""The branch-free division and square root of the Riemann solvers and the
limiter.

The kernels divide and take square roots with FastRn
(pyclaw_b200/csrc/claw2_fastrn.cuh): a Newton-Raphson result plus a proof,
from the exact FMA remainder, that it is the correctly rounded one; a tile
whose proofs did not all pass is redone with IEEE arithmetic.  These tests call
both operations on the GPU through claw2_fastrn_check and require, over many
millions of operands (random over the whole exponent range, typical solver
magnitudes and the hard cases), that every result marked as proven equals the
IEEE result bit for bit (numpy's division and square root on the host), that
the proof fails for every operand outside its range, and that it passes for
nearly all operands of ordinary size.
"""
import ctypes

import numpy as np
import pytest

import gpu_helpers as H
from pyclaw_b200 import _lib

pytestmark = pytest.mark.gpu


def _fastrn(op, a, b=None):
    t = H.torch()
    lib = _lib.load()
    da = t.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    db = t.from_numpy(np.ascontiguousarray(b, dtype=np.float64)).cuda() if b is not None else None
    q = t.empty_like(da)
    ok = t.empty(da.shape, dtype=t.uint8, device='cuda')
    rc = lib.claw2_fastrn_check(op, ctypes.c_void_p(da.data_ptr()),
                                ctypes.c_void_p(db.data_ptr()) if db is not None else None,
                                ctypes.c_void_p(q.data_ptr()), ctypes.c_void_p(ok.data_ptr()), da.numel(),
                                H.stream())
    assert rc == 0, _lib.load().claw2_strerror(rc)
    t.cuda.synchronize()
    return q.cpu().numpy(), ok.cpu().numpy().astype(bool)


def _fastdiv(a, b):
    return _fastrn(0, a, b)


def _fastsqrt(x):
    return _fastrn(1, x)


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


def _check_sqrt(x):
    """Every proven root equals numpy's IEEE root bit for bit.  Returns the
    proven fraction and mask."""
    r, ok = _fastsqrt(x)
    with np.errstate(all='ignore'):
        ref = np.sqrt(x)
    bad = ok & (_bits(r) != _bits(ref))
    assert not bad.any(), (x[bad][:5], r[bad][:5], ref[bad][:5])
    return ok.mean(), ok


def test_sqrt_random_and_ordinary():
    rng = np.random.default_rng(31)
    n = 1 << 23
    for _ in range(3):
        _check_sqrt(np.abs(_random_doubles(rng, n, -1022, 1023)))
        _check_sqrt(_random_doubles(rng, n, -1022, 1023))           # half negative: never proven
    for lo, hi in ((1e-3, 1e3), (1e-12, 1e-6), (1e6, 1e12)):
        frac, _ = _check_sqrt(rng.uniform(lo, hi, n))
        assert frac > 1.0 - 1e-6, frac
    frac, _ = _check_sqrt(np.abs(_random_doubles(rng, n, -900, 1000)))
    assert frac > 1.0 - 1e-6, frac


def test_sqrt_hard_cases():
    """Perfect squares (exact roots), squares of doubles and their neighbours
    (roots next to a midpoint), arguments next to powers of four (roots next
    to a power of two) and all-ones significands."""
    rng = np.random.default_rng(37)
    n = 1 << 22
    m = rng.integers(1, 1 << 26, n).astype(np.float64)
    scale = np.ldexp(1.0, 2 * rng.integers(-200, 200, n))
    frac, _ = _check_sqrt(m * m * scale)
    assert frac == 1.0
    s = np.abs(_random_doubles(rng, n, -300, 300))
    sq = s * s
    for x in (sq, np.nextafter(sq, np.inf), np.nextafter(sq, 0.0)):
        frac, _ = _check_sqrt(x)
        assert frac > 1.0 - 1e-6, frac
    k = rng.integers(0, 64, n, dtype=np.uint64)
    exp = rng.integers(1023 - 300, 1023 + 300, n).astype(np.uint64) << np.uint64(52)
    ones = np.uint64((1 << 52) - 1)
    for x in ((exp | k).view(np.float64), (exp | (ones - k)).view(np.float64)):
        frac, _ = _check_sqrt(x)
        assert frac > 0.9, frac      # roots next to a power of two use the smaller gap


def test_sqrt_specials_are_never_proven():
    tiny = np.nextafter(0.0, 1.0)
    x = np.array([0.0, -0.0, -1.0, -1e-300, tiny, 2.2250738585072014e-308, 2.0 ** -961, np.inf, -np.inf, np.nan])
    r, ok = _fastsqrt(x)
    assert not ok.any(), x[ok]
    x = np.array([2.0 ** -960, 1.0, 4.0, 2.0, 0.25])
    r, ok = _fastsqrt(x)
    assert ok.all()
    assert (_bits(r) == _bits(np.sqrt(x))).all()
    # the largest double: its root lies next to a midpoint below 2^512
    _check_sqrt(np.array([np.finfo(np.float64).max, np.nextafter(2.0 ** 1022, 0.0)]))
