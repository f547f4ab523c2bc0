"""Loader for libclaw2.so (the sm_100a CUDA library) and its C prototypes.

There is no fallback: if the library is missing or cannot be loaded, every
entry point that needs it raises ClawLibraryError.  The prototypes mirror
include/claw2.h and include/claw2_adjoint.h.
"""
import ctypes
import os

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclaw2.so")

# (name, restype, argtypes) for every function declared in include/*.h
_P = ctypes.POINTER(_abi.Problem)
_L = ctypes.POINTER(_abi.Layout)
_C = ctypes.POINTER(_abi.Control)
_dp = ctypes.c_void_p           # device or host double* (passed as an address)
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_dbl = ctypes.c_double

PROTOTYPES = [
    ("claw2_abi_version", ctypes.c_int, []),
    ("claw2_strerror", ctypes.c_char_p, [ctypes.c_int]),
    ("claw2_validate", ctypes.c_int, [_P]),
    ("claw2_get_layout", ctypes.c_int, [_P, _L]),
    ("claw2_scratch_bytes", ctypes.c_size_t, [_P]),
    ("claw2_fill_ghosts", ctypes.c_int, [_P, _dp, _vp]),
    ("claw2_fill_aux_ghosts", ctypes.c_int, [_P, _dp, _vp]),
    ("claw2_step", ctypes.c_int, [_P, _dp, _dp, _dp, _dbl, _vp, _dp, _vp]),
    ("claw2_step_noalloc", ctypes.c_int, [_P, _dp, _dp, _dp, _dbl, _dp, _vp]),
    ("claw2_debug_halo_shortfall", ctypes.c_int, [ctypes.c_int]),
    ("claw2_advance", ctypes.c_int, [_P, _dp, _dp, _dp, _vp, _vp, ctypes.c_int, _vp]),
    ("claw2_advance_hooked", ctypes.c_int, [_P, _dp, _dp, _dp, _vp, _vp, ctypes.c_int, ctypes.POINTER(_abi.Hooks),
                                            _vp]),
    ("claw2_advance_gauged", ctypes.c_int, [_P, _dp, _dp, _dp, _vp, _vp, ctypes.c_int, ctypes.POINTER(_abi.Hooks),
                                            ctypes.POINTER(_abi.Gauges), _vp]),
    ("claw2_step_ctrl", ctypes.c_int, [_P, _dp, _dp, _dp, _vp, _vp, _dp, _vp]),
    ("claw2_control_apply", ctypes.c_int, [_vp, _dp, _vp]),
    ("claw2_fill_ghosts_ctrl", ctypes.c_int, [_P, _dp, _dp, _vp, _vp]),
    ("claw2_halo_pack", ctypes.c_int, [_P, _dp, _dp, _vp, ctypes.c_int, _dp, _vp]),
    ("claw2_halo_unpack", ctypes.c_int, [_P, _dp, _dp, _vp, ctypes.c_int, _dp, _vp]),
    ("claw2_control_init", ctypes.c_int, [_C, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, ctypes.c_int,
                                          ctypes.c_int, _i64, _dbl]),
    ("claw2_ref_to_device", ctypes.c_int, [_P, ctypes.c_int, _dp, _dp, _vp]),
    ("claw2_device_to_ref", ctypes.c_int, [_P, ctypes.c_int, _dp, _dp, _vp]),
    ("claw2_batch_num_variants", ctypes.c_int, []),
    ("claw2_batch_variant_info", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_int)]),
    ("claw2_batch_tiles", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int)]),
    ("claw2_batch_variant_tile", ctypes.c_int, [ctypes.c_int]),
    ("claw2_batch_tiles_for", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                             ctypes.POINTER(ctypes.c_int)]),
    ("claw2_batch_advance", ctypes.c_int, [_P, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp]),
    ("claw2_batch_graph_create", ctypes.c_int, [_P, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.POINTER(_vp)]),
    ("claw2_batch_advance_map", ctypes.c_int, [_P, _vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int,
                                               _vp]),
    ("claw2_batch_graph_create_map", ctypes.c_int, [_P, _vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int,
                                                    ctypes.c_int, ctypes.POINTER(_vp)]),
    ("claw2_graph_launch", ctypes.c_int, [_vp, _vp]),
    ("claw2_graph_destroy", ctypes.c_int, [_vp]),
    ("claw2_session_create", ctypes.c_int, [_P, ctypes.POINTER(_vp)]),
    ("claw2_session_destroy", ctypes.c_int, [_vp]),
    ("claw2_session_step2", ctypes.c_int, [_vp, _dp, _dp, _dp, _dbl, ctypes.POINTER(_dbl)]),
    ("claw2_session_evolve", ctypes.c_int, [_vp, _dp, _dp, ctypes.POINTER(_dbl), ctypes.POINTER(_dbl),
                                            _dbl, _dbl, _dbl, _dbl, _i64, ctypes.POINTER(_dbl)]),
    # include/claw2_adjoint.h
    ("claw2_shots_scratch_bytes", ctypes.c_size_t, [_P, ctypes.c_int]),
    ("claw2_shots_step", ctypes.c_int, [_P, ctypes.c_int, _i64, _dp, _dp, _dp, _dbl, _vp, _dp, _vp]),
    ("claw2_shots_inject_record", ctypes.c_int, [_P, ctypes.c_int, _i64, _dp, _vp, _dp, ctypes.c_int, _vp, _dp,
                                                 _vp]),
    ("claw2_shots_adjoint_step", ctypes.c_int, [_P, ctypes.c_int, _i64, _dp, _dp, _dbl, _dp, _dp, _dp, _i64, _vp]),
    ("claw2_shots_adjoint_fold", ctypes.c_int, [_P, ctypes.c_int, _i64, _dp, ctypes.c_int, _vp, _dp, _vp]),
    ("claw2_shots_fold_aux", ctypes.c_int, [_P, ctypes.c_int, _i64, _dp, _vp]),
]


class ClawLibraryError(RuntimeError):
    """libclaw2.so is missing, unloadable, or a call into it failed."""


class ClawStatusError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        super().__init__("%s: %s (status %d)" % (what, _abi.STATUS_TEXT.get(code, "unknown"), code))


_LIB = None


def load():
    """Load libclaw2.so once; raise ClawLibraryError if it is not there."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ClawLibraryError(
            "libclaw2.so not found at %s; build it with `python -m pyclaw_b200.build` "
            "(needs nvcc with sm_100a support)" % LIB_PATH)
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        raise ClawLibraryError("cannot load %s: %s" % (LIB_PATH, e)) from e
    for name, res, args in PROTOTYPES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.claw2_abi_version() != _abi.ABI_VERSION:
        raise ClawLibraryError("libclaw2.so ABI %d != %d" % (lib.claw2_abi_version(), _abi.ABI_VERSION))
    _LIB = lib
    return lib


def check(rc, what):
    if rc != 0:
        raise ClawStatusError(rc, what)
    return rc


def layout(p):
    L = _abi.Layout()
    check(load().claw2_get_layout(ctypes.byref(p), ctypes.byref(L)), "claw2_get_layout")
    return L
