"""The allocation-free step entry point (claw2_step_noalloc).

Callers that may not allocate GPU memory -- because their device memory is a
pool they manage themselves, because their time loop must not call the CUDA
allocator, or because their language binding can hand over pointers but not
own device allocations -- step through claw2_step_noalloc, whose scratch is a
static array inside libclaw2.so.  This file sorts last so that a run stopping
at the first failure has already run every other test; it also passes alone in
a fresh process, where the first call performs the per-device set-up.

Every solver body keeps its CFL partials in that array, one per tile, so the
cases cover each body and tile size: the lean body (Euler, 28x28 tiles), the
generic split body, and the light acoustics body on its 13x13 small-grid tiles
and on its 29x29 tiles, with and without aux arrays, and a problem of exactly
CLAW2_NOALLOC_MAX_TILES tiles.  Results must equal claw2_step's (the entry
point with caller-provided scratch) bit for bit on two calls in a row.
"""
import ctypes

import numpy as np
import pytest

import gpu_helpers as H
from pyclaw_b200 import _abi, _lib

pytestmark = pytest.mark.gpu

NOALLOC_MAX_TILES = 32768          # CLAW2_NOALLOC_MAX_TILES in include/claw2.h


def _noalloc_step(p, qbc, auxbc, dt):
    t = H.torch()
    lib = _lib.load()
    L = _lib.layout(p)
    qin = H.to_dev(p, qbc, L)
    qout = t.full_like(qin, float('nan'))
    aux = H.to_dev(p, auxbc, L) if auxbc is not None else None
    cfl = t.zeros(1, dtype=t.float64, device='cuda')
    rc = lib.claw2_step_noalloc(ctypes.byref(p), ctypes.c_void_p(qin.data_ptr()), ctypes.c_void_p(qout.data_ptr()),
                                ctypes.c_void_p(aux.data_ptr()) if aux is not None else None, float(dt),
                                ctypes.c_void_p(cfl.data_ptr()), H.stream())
    _lib.check(rc, "claw2_step_noalloc")
    t.cuda.synchronize()
    return H.from_dev(p, qout, p.num_eqn, L), float(cfl.item())


def _two_calls(orc, p, dt, seed):
    q, aux = H.init_fields(p, seed=seed)
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    auxbc = None
    if aux is not None:
        auxbc = orc.new_qbc(p, aux, ncomp=p.num_aux)
        orc.fill_aux_ghosts(p, auxbc)
    for call in range(2):
        ref, cfl_ref = H.dev_step(p, qbc, auxbc, dt)        # caller-provided scratch
        got, cfl = _noalloc_step(p, qbc, auxbc, dt)
        assert cfl == cfl_ref, (call, cfl, cfl_ref)
        assert np.array_equal(got, ref), (call, np.nanmax(np.abs(got - ref)))
        qbc = np.asfortranarray(ref)                         # next call continues from the result


@pytest.mark.parametrize("tr", [2, -1])
def test_noalloc_step_equals_claw2_step_on_two_calls_in_a_row(orc, tr):
    p = H.problem("euler4", 97, 71, tr, bcl=(1, 3), bcu=(1, 3))
    _two_calls(orc, p, 0.002, seed=11)


# 60 x 50: 6 tiles of 29x29, under 148, so the light body runs 13x13 tiles
# (5 x 4 = 20 partials); 300 x 180: 11 x 7 = 77 tiles of 29 is still small;
# 480 x 420: 17 x 15 = 255 tiles of 29x29.
@pytest.mark.parametrize("name", ["acoustics", "vc_acoustics"])
@pytest.mark.parametrize("shape", [(60, 50), (300, 180), (480, 420)])
def test_noalloc_light_body_on_small_and_large_tiles(orc, name, shape):
    mx, my = shape
    p = H.problem(name, mx, my, 2, bcl=(3, 1), bcu=(1, 3))
    _two_calls(orc, p, 0.3 / max(mx, my), seed=mx + my)


def test_noalloc_accepts_exactly_its_maximum():
    """29 x 256 by 29 x 128 cells of acoustics: 256 x 128 = 32768 tiles of 29x29."""
    t = H.torch()
    lib = _lib.load()
    mx, my = 29 * 256, 29 * 128
    p = H.problem("acoustics", mx, my, 2, bcl=(3, 3), bcu=(3, 3))
    nbx, nby = (mx + 28) // 29, (my + 28) // 29
    assert nbx * nby == NOALLOC_MAX_TILES
    assert lib.claw2_scratch_bytes(ctypes.byref(p)) == 64 + 8 * NOALLOC_MAX_TILES
    L = _lib.layout(p)
    dev = t.device('cuda')
    qin = t.zeros(3 * L.plane, dtype=t.float64, device=dev)
    x = (t.arange(mx, dtype=t.float64, device=dev) + 0.5) / mx
    y = (t.arange(my, dtype=t.float64, device=dev) + 0.5) / my
    r2 = (x[None, :] - 0.4) ** 2 + (y[:, None] - 0.6) ** 2
    planes = qin.view(3, L.rows, L.ld)
    planes[0, 2:my + 2, 2:mx + 2] = t.exp(-200.0 * r2)
    planes[1, 2:my + 2, 2:mx + 2] = 0.1 * t.sin(7.0 * x)[None, :]
    _lib.check(lib.claw2_fill_ghosts(ctypes.byref(p), ctypes.c_void_p(qin.data_ptr()), H.stream()),
               "claw2_fill_ghosts")
    scratch = t.zeros(lib.claw2_scratch_bytes(ctypes.byref(p)), dtype=t.uint8, device=dev)
    dt = 0.4 / mx
    for call in range(2):
        ref = t.zeros_like(qin)
        got = t.zeros_like(qin)
        cfl_ref = t.zeros(1, dtype=t.float64, device=dev)
        cfl = t.zeros(1, dtype=t.float64, device=dev)
        _lib.check(lib.claw2_step(ctypes.byref(p), ctypes.c_void_p(qin.data_ptr()), ctypes.c_void_p(ref.data_ptr()),
                                  None, dt, ctypes.c_void_p(scratch.data_ptr()), ctypes.c_void_p(cfl_ref.data_ptr()),
                                  H.stream()), "claw2_step")
        _lib.check(lib.claw2_step_noalloc(ctypes.byref(p), ctypes.c_void_p(qin.data_ptr()),
                                          ctypes.c_void_p(got.data_ptr()), None, dt,
                                          ctypes.c_void_p(cfl.data_ptr()), H.stream()), "claw2_step_noalloc")
        t.cuda.synchronize()
        assert float(cfl.item()) == float(cfl_ref.item()) and float(cfl.item()) > 0.0
        assert t.equal(got, ref), call
        qin = ref
    del qin, got, ref, planes, scratch
    t.cuda.empty_cache()


def test_noalloc_rejects_problems_beyond_its_maximum():
    lib = _lib.load()
    n = 29 * 182                       # 182 x 182 = 33124 tiles > CLAW2_NOALLOC_MAX_TILES
    p = H.problem("acoustics", n, n, 2)
    rc = lib.claw2_step_noalloc(ctypes.byref(p), ctypes.c_void_p(16), ctypes.c_void_p(32), None, 0.1,
                                ctypes.c_void_p(64), H.stream())
    assert rc == _abi.ERR_SIZE
