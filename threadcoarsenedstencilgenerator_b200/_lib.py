"""ctypes binding of libtcs.so (the C ABI declared in include/tcs.h).

The library is built in-tree by ``threadcoarsenedstencilgenerator_b200.build``; when it is
missing this module raises instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtcs.so"

TCS_OK = 0
TCS_ERR_INVALID_VALUE = 1
TCS_ERR_CUDA = 2
TCS_ERR_COMPILE = 3
TCS_ERR_UNSUPPORTED = 4
TCS_ERR_DEVICE_TIMEOUT = 5
TCS_ERR_NO_DEVICE = 6

VARIANT_AUTO = 0
VARIANT_DIRECT = 1
VARIANT_MARCH = 2
VARIANT_PIPE = 3

LAUNCH_SHUFFLE = 1
LAUNCH_NO_SHUFFLE = 2
LAUNCH_TMEM = 4
LAUNCH_LOCKSTEP = 8


class TcsError(RuntimeError):
    """A libtcs call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__("[tcs %d] %s" % (code, message))
        self.code = code


class CudaErrorInvalidValue(TcsError):
    """Raised where the reference throws ``cudaErrorInvalidValue`` (parameter mismatch)."""


class UnsupportedLaunch(TcsError):
    """The requested kernel variant cannot run this launch shape."""


class CSpec(ctypes.Structure):
    _fields_ = [
        ("dimension", ctypes.c_int),
        ("neighbourhood", ctypes.c_int),
        ("orientation", ctypes.c_int),
        ("coefficients", ctypes.c_int),
        ("range", ctypes.c_int),
        ("cx", ctypes.c_int),
        ("cy", ctypes.c_int),
        ("cz", ctypes.c_int),
        ("alignment", ctypes.c_int),
        ("cl_size", ctypes.c_int),
        ("precision", ctypes.c_int),
    ]


class CGeometry(ctypes.Structure):
    _fields_ = [
        ("grid", ctypes.c_uint * 3),
        ("elements", ctypes.c_uint * 3),
        ("threads", ctypes.c_uint * 3),
        ("left_offset", ctypes.c_uint),
        ("right_offset", ctypes.c_uint),
        ("n_points", ctypes.c_ulonglong),
    ]


class CLaunch(ctypes.Structure):
    _fields_ = [
        ("block", ctypes.c_uint * 3),
        ("grid_blocks", ctypes.c_uint * 3),
        ("variant", ctypes.c_int),
        ("segments", ctypes.c_uint),
        ("depth", ctypes.c_uint),
        ("chunk", ctypes.c_uint),
        ("flags", ctypes.c_uint),
    ]


class CPlan(ctypes.Structure):
    _fields_ = [
        ("variant", ctypes.c_int),
        ("grid_blocks", ctypes.c_uint * 3),
        ("block", ctypes.c_uint * 3),
        ("dyn_smem", ctypes.c_uint),
        ("seg_len", ctypes.c_uint),
        ("nslot", ctypes.c_uint),
        ("width", ctypes.c_uint),
        ("chunk", ctypes.c_uint),
        ("depth", ctypes.c_uint),
        ("loader", ctypes.c_uint),
        ("ctas_per_sm", ctypes.c_int),
        ("num_sms", ctypes.c_int),
    ]


U3 = ctypes.c_uint * 3
_P = ctypes.POINTER
_vp = ctypes.c_void_p
_u = ctypes.c_uint
_i = ctypes.c_int

# name -> argtypes (all return int status unless listed in _RESTYPE)
SIGNATURES = {
    "tcs_abi_version": [],
    "tcs_last_error": [],
    "tcs_spec_validate": [_P(CSpec)],
    "tcs_stencil_size": [_P(CSpec), _P(_u), _P(_u)],
    "tcs_compute_geometry": [_P(CSpec), _u, _u, _u, _P(CGeometry)],
    "tcs_compute_geometry_ragged": [_P(CSpec), _u, _u, _u, _P(CGeometry)],
    "tcs_left_offset": [_P(CSpec), _P(_u)],
    "tcs_create": [_P(CSpec), _P(_vp)],
    "tcs_destroy": [_vp],
    "tcs_get_spec": [_vp, _P(CSpec)],
    "tcs_copy_mask": [_vp, _P(ctypes.c_double), _u],
    "tcs_max_potential_block_size": [_vp, _P(_i)],
    "tcs_plan_launch": [_vp, U3, _u, _P(CLaunch), _P(CPlan)],
    "tcs_update_grid": [_vp, U3, _u, _P(CLaunch), _vp, _vp, _vp],
    "tcs_sweeps": [_vp, U3, _u, _P(CLaunch), _vp, _vp, _u, _vp, _P(_i)],
    "tcs_time_sweeps": [_vp, U3, _u, _P(CLaunch), _vp, _vp, _u, _vp, _P(ctypes.c_float)],
    "tcs_sweep_host_jobs": [_vp, U3, _u, _P(CLaunch), _P(_vp), _P(_vp), _u, _u, _P(_vp), _P(_vp), _u,
                            _P(ctypes.c_float)],
    "tcs_benchmark_update_grid": [_vp, ctypes.c_char_p, ctypes.c_char_p, _u, _u, ctypes.c_char_p,
                                  ctypes.c_double, U3, U3, U3, _vp, _vp, _u, _P(ctypes.c_double), _u,
                                  _P(_u)],
    "tcs_launch_init": [_vp, U3, U3, U3, _vp, _u],
    "tcs_device_status": [_vp, _P(_u), _i],
    "tcs_self_test_wait": [_vp, ctypes.c_longlong],
    "tcs_set_dropin_launch": [_vp, _i, _u, _u],
    "tcs_precompile": [_P(CSpec), ctypes.c_char_p, _u],
    "tcs_precompile_pipe": [_P(CSpec), _u, _u, _u, ctypes.c_char_p, _u],
    "tcs_update_grid_source": [_vp, U3, _u, _P(CLaunch), _vp, _vp, _vp, _vp],
    "tcs_residual": [_vp, U3, _u, _vp, _vp, _vp, _P(ctypes.c_double), _vp],
    "tcs_residual_static": [_vp, U3, _u, _vp, _vp, _vp, _P(ctypes.c_double), _u, _vp],
    "tcs_defect_sweep": [_vp, U3, _u, _P(CLaunch), _vp, _vp, _P(ctypes.c_double), _vp],
    "tcs_update_grid_accumulate": [_vp, U3, _u, _P(CLaunch), _vp, _vp, _vp, _vp],
    "tcs_precompile_pipe_epilogue": [_P(CSpec), _u, _u, _u, _u, ctypes.c_char_p, _u],
    "tcs_precompile_pipe_flags": [_P(CSpec), _u, _u, _u, _u, ctypes.c_char_p, _u],
    "tcs_sweeps_tb3": [_vp, U3, _u, _P(CLaunch), _vp, _vp, _u, _vp, _P(ctypes.c_int)],
    "tcs_plan_tb3": [_vp, U3, _u, _P(CLaunch), _P(CPlan)],
    "tcs_precompile_tb3": [_P(CSpec), _u, _u, _u, ctypes.c_char_p, _u],
    "tcs_scratch_bytes": [_vp, _P(ctypes.c_ulonglong)],
    "tcs_benchmark_durations": [_vp, _vp, _u, _P(_u)],
    "tcs_accumulate": [_vp, U3, _u, _vp, _vp, _vp],
    "tcs_compare": [_vp, U3, _u, _vp, _i, _vp, _P(ctypes.c_double), _vp],
    "tcs_device_sm_count": [_P(_i)],
    "tcs_batch_create": [_vp, _u, _P(_u), _P(_u), _P(CLaunch), _P(_vp), _P(_vp), _P(_vp)],
    "tcs_batch_plan": [_vp, _P(CPlan)],
    "tcs_batch_sweep": [_vp, _i, _vp],
    "tcs_batch_sweep_separate": [_vp, _i, _vp],
    "tcs_batch_graph": [_vp, _u, _i],
    "tcs_batch_graph_launch": [_vp, _vp],
    "tcs_batch_destroy": [_vp],
    "tcs_precompile_batch": [_P(CSpec), _u, _u, _u, ctypes.c_char_p, _u],
    "tcs_mlp_create": [_u, _u, _u, _P(_vp)],
    "tcs_mlp_param_count": [_vp, _P(_u)],
    "tcs_mlp_set_params": [_vp, _P(ctypes.c_float), _u],
    "tcs_mlp_get_params": [_vp, _P(ctypes.c_float), _u],
    "tcs_mlp_forward": [_vp, _vp, _u, _vp, _vp],
    "tcs_mlp_gradient": [_vp, _vp, _vp, _u, _vp, _P(ctypes.c_float), _vp],
    "tcs_mlp_adam_step": [_vp, _vp, _vp, _u, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                          _P(ctypes.c_float), _vp],
    "tcs_mlp_destroy": [_vp],
    "tcs_sweeps_tb2": [_vp, U3, _u, _vp, _vp, _u, _vp, _P(_i)],
    "tcs_precompile_fringe": [_P(CSpec), ctypes.c_char_p, _u],
    "tcs_tc_supported": [_P(CSpec)],
    "tcs_tc_update_grid": [_vp, U3, _u, _vp, _vp, _vp, _vp],
}
_RESTYPE = {"tcs_last_error": ctypes.c_char_p}

_lib = None


def load() -> ctypes.CDLL:
    """Load libtcs.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                "libtcs.so is missing: build it with `python -m threadcoarsenedstencilgenerator_b200.build`"
            )
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, argtypes in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = lib
    return _lib


def last_error() -> str:
    msg = load().tcs_last_error()
    return msg.decode(errors="replace") if msg else ""


def check(rc: int) -> None:
    if rc == TCS_OK:
        return
    msg = last_error()
    if rc == TCS_ERR_INVALID_VALUE:
        raise CudaErrorInvalidValue(rc, msg)
    if rc == TCS_ERR_UNSUPPORTED:
        raise UnsupportedLaunch(rc, msg)
    raise TcsError(rc, msg)
