"""The domain decomposition's CUDA kernels (halo pack/unpack, the step that
reports its CFL, the controller update from the reduced CFL, the ghost fill
of the current buffer) on one GPU: several slabs driven by one process with
decomp.LocalTransport (halo exchange = device copy; no kernel waits on
another) equal the single-grid run bit for bit."""
import ctypes

import numpy as np
import pytest

import decomp_helpers as D
from pyclaw_b200 import _abi, _lib, decomp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case,n", [("euler_case", 2), ("euler_case", 3), ("vc_case", 2), ("vc_case", 4)])
def test_slabs_on_one_gpu_equal_single_domain(case, n):
    p, q, aux, run = getattr(D, case)()
    lib = _lib.load()
    c = _abi.Control()
    _lib.check(lib.claw2_control_init(ctypes.byref(c), 0.0, run["dt_initial"], run["tend"], run["cfl_max"],
                                      run["cfl_desired"], 1e99, 1, 0, 1 << 40, run["cfl_desired"]),
               "claw2_control_init")
    slabs = [decomp.Slab(p, n, r) for r in range(n)]
    for s in slabs:
        s.upload(q, aux)
        s.init_control(c)
    out = decomp.evolve(slabs, decomp.LocalTransport(slabs), batch=4)
    got = np.concatenate([s.solution() for s in slabs], axis=2)
    ref, ctrl = D.single_domain(p, q, aux, run)
    assert np.array_equal(got, ref), np.max(np.abs(got - ref))
    assert out.numsteps == ctrl.numsteps and out.t == ctrl.t and out.error == 0
    assert all(s.control().numsteps == out.numsteps for s in slabs)
