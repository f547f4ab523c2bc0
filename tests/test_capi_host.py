"""Host-side checks of the C ABI (no GPU needed): the library loads, exports
every function include/*.h declares, and its host-only entry points
(validation, layout, scratch size, controller initialisation) behave."""
import ctypes
import os
import re

import numpy as np
import pytest

from pyclaw_b200 import _abi, _lib
import gpu_helpers as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for h in sorted(os.listdir(inc)):
        if h.endswith(".h"):
            with open(os.path.join(inc, h)) as f:
                names.update(re.findall(r"CLAW2_EXPORT\s+(?:const\s+)?\w+\*?\s+(claw2_\w+)\s*\(", f.read()))
    return sorted(names)


def test_header_declares_the_prototypes_python_binds():
    names = declared_functions()
    assert len(names) >= 15
    assert sorted(n for n, _, _ in _lib.PROTOTYPES) == names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.claw2_abi_version() == _abi.ABI_VERSION
    assert lib.claw2_strerror(_abi.ERR_CFL) == b"CFL too large, giving up!"


def test_validate_and_layout():
    lib = _lib.load()
    p = H.problem("euler4", 1280, 320, 2)
    assert lib.claw2_validate(ctypes.byref(p)) == 0
    L = _lib.layout(p)
    assert L.ld % 16 == 0 and L.ld >= 1284 and L.rows == 324
    assert L.plane == L.ld * L.rows and L.q_elems == 4 * L.plane
    # a 64-byte header and one double per CTA: the unsplit Euler step runs
    # 28 x 28 tiles (lean body), the split step 28 x 28, the acoustics bodies
    # 29 x 29 (13 x 13 on grids of fewer than 148 such tiles)
    nb = lib.claw2_scratch_bytes(ctypes.byref(p))
    nt = ((1280 + 27) // 28) * ((320 + 27) // 28)
    assert nb == 64 + 8 * nt
    ps = H.problem("euler4", 1280, 320, -1)
    assert lib.claw2_scratch_bytes(ctypes.byref(ps)) == 64 + 8 * nt
    pa = H.problem("acoustics", 1280, 320, 2)
    assert lib.claw2_scratch_bytes(ctypes.byref(pa)) == 64 + 8 * ((1280 + 28) // 29) * ((320 + 28) // 29)
    pa = H.problem("acoustics", 256, 256, 2)
    assert lib.claw2_scratch_bytes(ctypes.byref(pa)) == 64 + 8 * ((256 + 12) // 13) ** 2
    bad = H.problem("euler4", 64, 64, 2)
    bad.num_eqn = 3
    assert lib.claw2_validate(ctypes.byref(bad)) == _abi.ERR_INVALID
    per = H.problem("acoustics", 64, 64, 2, bcl=(2, 1), bcu=(1, 1))
    assert lib.claw2_validate(ctypes.byref(per)) == _abi.ERR_UNSUPPORTED
    neg = H.problem("acoustics", 64, 64, 2, mthlim=(-1,))
    assert lib.claw2_validate(ctypes.byref(neg)) == _abi.ERR_INVALID


@pytest.mark.parametrize("args", [
    (0.0, 0.1, 0.6, 1.0, 0.9, 1e99, 1, 0, 10000, 0.9),
    (0.55, 0.1, 0.6, 1.0, 0.9, 1e99, 1, 0, 10000, 0.3),      # clamp to tend
    (0.0, 0.1, 0.3, 1.0, 0.9, 1e99, 0, 0, 10000, 0.9),       # fixed dt
    (0.0, 0.1, 0.0, 1.0, 0.9, 1e99, 1, 0, 10000, 0.9),       # already at tend
    (0.0, 0.1, 0.0, 1.0, 0.9, 1e99, 1, 1, 10000, 0.9),       # one step
])
def test_control_init_matches_oracle(orc, args):
    lib = _lib.load()
    c = _abi.Control()
    rc = lib.claw2_control_init(ctypes.byref(c), *args)
    o = _abi.Control()
    rco = orc.load().orc_control_init(ctypes.byref(o), *args)
    assert rc == rco
    assert bytes(c) == bytes(o)


def test_control_init_rejects_like_the_reference():
    lib = _lib.load()
    c = _abi.Control()
    # fixed dt that does not divide the interval (solver.py:622-624)
    assert lib.claw2_control_init(ctypes.byref(c), 0.0, 0.07, 0.3, 1.0, 0.9, 1e99, 0, 0, 100, 0.9) != 0
    # cfl_desired > cfl_max with variable dt (:625-626)
    assert lib.claw2_control_init(ctypes.byref(c), 0.0, 0.1, 0.3, 0.5, 0.9, 1e99, 1, 0, 100, 0.9) != 0


def test_missing_gpu_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from pyclaw_b200.device import DeviceState
    p = H.problem("euler4", 16, 16, 2)
    with pytest.raises(_lib.ClawLibraryError):
        DeviceState(p)
