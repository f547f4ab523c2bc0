"""The allocation-free step entry point (claw2_step_noalloc).

Callers that may not allocate GPU memory -- because their device memory is a
pool they manage themselves, because their time loop must not call the CUDA
allocator, or because their language binding can hand over pointers but not
own device allocations -- step through claw2_step_noalloc, whose scratch is a
static array inside libclaw2.so.  This file sorts last so that a run stopping
at the first failure has already run every other test; it also passes alone in
a fresh process, where the first call performs the per-device set-up.
"""
import ctypes

import numpy as np
import pytest

import gpu_helpers as H
from pyclaw_b200 import _abi, _lib

pytestmark = pytest.mark.gpu


def _noalloc_step(p, qbc, dt):
    t = H.torch()
    lib = _lib.load()
    L = _lib.layout(p)
    qin = H.to_dev(p, qbc, L)
    qout = t.full_like(qin, float('nan'))
    cfl = t.zeros(1, dtype=t.float64, device='cuda')
    rc = lib.claw2_step_noalloc(ctypes.byref(p), ctypes.c_void_p(qin.data_ptr()), ctypes.c_void_p(qout.data_ptr()),
                                None, float(dt), ctypes.c_void_p(cfl.data_ptr()), H.stream())
    _lib.check(rc, "claw2_step_noalloc")
    t.cuda.synchronize()
    return H.from_dev(p, qout, p.num_eqn, L), float(cfl.item())


@pytest.mark.parametrize("tr", [2, -1])
def test_noalloc_step_equals_claw2_step_on_two_calls_in_a_row(orc, tr):
    p = H.problem("euler4", 97, 71, tr, bcl=(1, 3), bcu=(1, 3))
    q, _ = H.init_fields(p, seed=11)
    qbc = orc.new_qbc(p, q)
    orc.fill_ghosts(p, qbc)
    for call in range(2):
        ref, cfl_ref = H.dev_step(p, qbc, None, 0.002)      # caller-provided scratch
        got, cfl = _noalloc_step(p, qbc, 0.002)
        assert cfl == cfl_ref, (call, cfl, cfl_ref)
        assert np.array_equal(got, ref), (call, np.nanmax(np.abs(got - ref)))
        qbc = np.asfortranarray(ref)                         # next call continues from the result


def test_noalloc_rejects_problems_beyond_its_maximum():
    lib = _lib.load()
    n = 29 * 182                       # 182 x 182 = 33124 tiles > CLAW2_NOALLOC_MAX_TILES
    p = H.problem("acoustics", n, n, 2)
    rc = lib.claw2_step_noalloc(ctypes.byref(p), ctypes.c_void_p(16), ctypes.c_void_p(32), None, 0.1,
                                ctypes.c_void_p(64), H.stream())
    assert rc == _abi.ERR_SIZE
