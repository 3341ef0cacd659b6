"""CPU oracle for the stencil engine — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
this package, and only as the checker (or as the timed CPU baseline).  The engine
(``threadcoarsenedstencilgenerator_b200``) never imports it and has no CPU fallback.

``stencil_oracle.c`` restates the reference generator's kernel arithmetic in C (file:line
citations in its header); ``build.py`` compiles it into ``oracle/liboracle.so``.  The wrappers
below take and return numpy arrays laid out like the reference's device buffers: ``[y][x]`` (2D)
or ``[z][y][x]`` (3D) with the padded row pitch as the last extent.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .build import LIB_PATH, build_oracle

_lib = None


class OracleSpec(ctypes.Structure):
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
    ]


class OracleGeometry(ctypes.Structure):
    _fields_ = [
        ("grid", ctypes.c_uint * 3),
        ("elements", ctypes.c_uint * 3),
        ("threads", ctypes.c_uint * 3),
        ("left_offset", ctypes.c_uint),
        ("right_offset", ctypes.c_uint),
        ("n_points", ctypes.c_ulonglong),
    ]


_SHAPES = {"Box": 0, "Star": 1}
_ORIENTS = {"Row": 0, "Column": 1}
_COEFFS = {"Jacobi": 0, "Variable": 1}
_ALIGNS = {"None": 0, "Read": 1, "Write": 2}


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build_oracle()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.POINTER
        u3 = ctypes.c_uint * 3
        for name, T in (("f64", ctypes.c_double), ("f32", ctypes.c_float)):
            f = getattr(L, "oracle_sweep_" + name)
            f.argtypes = [P(OracleSpec), u3, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            f.restype = ctypes.c_int
            f = getattr(L, "oracle_cpu_sweep_" + name)
            f.argtypes = [P(OracleSpec), u3, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
            f.restype = ctypes.c_int
        L.oracle_geometry_of.argtypes = [P(OracleSpec), ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, P(OracleGeometry)]
        L.oracle_term_order.argtypes = [P(OracleSpec), ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_init_f64.argtypes = [P(OracleSpec), u3, ctypes.c_uint, ctypes.c_void_p]
        L.oracle_stencil_size.argtypes = [P(OracleSpec)]
        _lib = L
    return _lib


def make_spec(dimension, neighbourhood, orientation, coefficients, range_, cx, cy, cz=1,
              alignment="None", cl_size=0) -> OracleSpec:
    return OracleSpec(int(dimension), _SHAPES[neighbourhood], _ORIENTS[orientation], _COEFFS[coefficients],
                      int(range_), int(cx), int(cy), int(cz) if int(dimension) == 3 else 1,
                      _ALIGNS[alignment], int(cl_size))


@dataclass
class Geometry:
    grid: tuple
    elements: tuple
    threads: tuple
    left_offset: int
    right_offset: int
    n_points: int


def geometry(spec: OracleSpec, nx: int, ny: int, nz: int = 1) -> Geometry:
    g = OracleGeometry()
    rc = lib().oracle_geometry_of(ctypes.byref(spec), nx, ny, nz, ctypes.byref(g))
    if rc:
        raise ValueError("grid smaller than twice the stencil range")
    return Geometry(tuple(g.grid), tuple(g.elements), tuple(g.threads), g.left_offset, g.right_offset,
                    g.n_points)


def stencil_size(spec: OracleSpec) -> int:
    return lib().oracle_stencil_size(ctypes.byref(spec))


def term_order(spec: OracleSpec):
    """Per-output term order as (offsets[S,3], mask_index[S])."""
    S = stencil_size(spec)
    off = np.zeros((S, 3), dtype=np.int32)
    mi = np.zeros(S, dtype=np.int32)
    n = lib().oracle_term_order(ctypes.byref(spec), off.ctypes.data, mi.ctypes.data)
    assert n == S
    return off, mi


def _grid_of(spec: OracleSpec, a: np.ndarray):
    if spec.dimension == 2:
        assert a.ndim == 2
        return (ctypes.c_uint * 3)(a.shape[1], a.shape[0], 1)
    assert a.ndim == 3
    return (ctypes.c_uint * 3)(a.shape[2], a.shape[1], a.shape[0])


def _mask_arg(spec: OracleSpec, mask, dtype):
    S = stencil_size(spec)
    if spec.coefficients == 0:
        m = np.zeros(S, dtype=dtype)
    else:
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.float64).astype(dtype))
        assert m.size == S
    return m


def sweep(spec: OracleSpec, a: np.ndarray, right_offset: int = 0, mask=None, out: np.ndarray | None = None):
    """One reference sweep of ``a`` (float64 or float32); points outside the interior are
    copied from ``out`` if given, else from ``a``."""
    a = np.ascontiguousarray(a)
    dt = a.dtype
    assert dt in (np.float64, np.float32)
    o = a.copy() if out is None else out
    m = _mask_arg(spec, mask, dt)
    f = lib().oracle_sweep_f64 if dt == np.float64 else lib().oracle_sweep_f32
    rc = f(ctypes.byref(spec), _grid_of(spec, a), right_offset, a.ctypes.data, o.ctypes.data, m.ctypes.data)
    assert rc == 0
    return o


def cpu_sweep(spec: OracleSpec, a: np.ndarray, out: np.ndarray, right_offset: int = 0, mask=None,
              threads: int = 0) -> None:
    """OpenMP sweep in the same term order (the timed CPU baseline); writes the interior of out."""
    dt = a.dtype
    m = _mask_arg(spec, mask, dt)
    f = lib().oracle_cpu_sweep_f64 if dt == np.float64 else lib().oracle_cpu_sweep_f32
    rc = f(ctypes.byref(spec), _grid_of(spec, a), right_offset, a.ctypes.data, out.ctypes.data,
           m.ctypes.data, int(threads))
    assert rc == 0


def sweeps(spec: OracleSpec, a: np.ndarray, n: int, right_offset: int = 0, mask=None, cpu_threads: int | None = None):
    """n ping-pong sweeps; both buffers start as ``a`` (fixed Dirichlet border)."""
    x = np.ascontiguousarray(a).copy()
    y = x.copy()
    for _ in range(n):
        if cpu_threads is None:
            sweep(spec, x, right_offset, mask, out=y)
        else:
            cpu_sweep(spec, x, y, right_offset, mask, cpu_threads)
        x, y = y, x
    return x


def init_pattern(spec: OracleSpec, grid, right_offset: int, fill: float = np.nan) -> np.ndarray:
    """The reference's init kernel applied to a buffer pre-filled with ``fill``."""
    if spec.dimension == 2:
        a = np.full((grid[1], grid[0]), fill, dtype=np.float64)
    else:
        a = np.full((grid[2], grid[1], grid[0]), fill, dtype=np.float64)
    lib().oracle_init_f64(ctypes.byref(spec), (ctypes.c_uint * 3)(*grid), right_offset, a.ctypes.data)
    return a


def max_threads() -> int:
    return lib().oracle_max_threads()
