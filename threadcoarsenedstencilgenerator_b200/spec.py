"""Stencil parameter set and grid geometry.

``StencilSpec`` is the parameter surface of the reference's generators
(cuda/generate2DStencil_cuda.py:15-60, cuda/generate3DStencil_cuda.py:15-63) plus the element
precision.  Validation, stencil size, flops and geometry are answered by libtcs.so's host-only
entry points, which follow cuda/benchmark.cpp:62-81,142-179,430-491 and cuda/benchmark.h:100-123.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import _lib

NEIGHBOURHOODS = ("Box", "Star")
ORIENTATIONS = ("Row", "Column")
COEFFICIENTS = ("Jacobi", "Variable")
ALIGNMENTS = ("None", "Read", "Write")
PRECISIONS = ("f64", "f32", "f32c")  # f32c: FP32 grids, compensated (two-sum) accumulation


@dataclass(frozen=True)
class StencilSpec:
    dimension: int = 2
    neighbourhood: str = "Box"
    orientation: str = "Row"
    coefficients: str = "Jacobi"
    range: int = 1
    cx: int = 1
    cy: int = 1
    cz: int = 1
    alignment: str = "None"
    cl_size: int = 0
    precision: str = "f64"

    def __post_init__(self):
        for name, allowed in (("neighbourhood", NEIGHBOURHOODS), ("orientation", ORIENTATIONS),
                              ("coefficients", COEFFICIENTS), ("alignment", ALIGNMENTS),
                              ("precision", PRECISIONS)):
            if getattr(self, name) not in allowed:
                raise _lib.CudaErrorInvalidValue(
                    _lib.TCS_ERR_INVALID_VALUE, "Unknown %s: %r (one of %s)" % (name, getattr(self, name), allowed))
        if self.dimension == 2 and self.cz != 1:
            object.__setattr__(self, "cz", 1)
        _lib.check(_lib.load().tcs_spec_validate(ctypes.byref(self.to_c())))

    def to_c(self) -> _lib.CSpec:
        return _lib.CSpec(
            int(self.dimension), NEIGHBOURHOODS.index(self.neighbourhood), ORIENTATIONS.index(self.orientation),
            COEFFICIENTS.index(self.coefficients), int(self.range), int(self.cx), int(self.cy),
            int(self.cz) if self.dimension == 3 else 1, ALIGNMENTS.index(self.alignment), int(self.cl_size),
            PRECISIONS.index(self.precision))

    @property
    def stencil_size(self) -> int:
        s, f = ctypes.c_uint(), ctypes.c_uint()
        _lib.check(_lib.load().tcs_stencil_size(ctypes.byref(self.to_c()), ctypes.byref(s), ctypes.byref(f)))
        return s.value

    @property
    def flops_per_update(self) -> int:
        s, f = ctypes.c_uint(), ctypes.c_uint()
        _lib.check(_lib.load().tcs_stencil_size(ctypes.byref(self.to_c()), ctypes.byref(s), ctypes.byref(f)))
        return f.value

    @property
    def left_offset(self) -> int:
        v = ctypes.c_uint()
        _lib.check(_lib.load().tcs_left_offset(ctypes.byref(self.to_c()), ctypes.byref(v)))
        return v.value

    @property
    def coarsening(self) -> tuple:
        return (self.cx, self.cy, self.cz if self.dimension == 3 else 1)

    @property
    def itemsize(self) -> int:
        return 8 if self.precision == "f64" else 4

    def geometry(self, nx: int, ny: int, nz: int = 1, ragged: bool = False) -> "Geometry":
        """The reference's geometry; ``ragged=True`` keeps the interior whole instead of truncating
        it to a coarsening multiple (sweeps then also update the partial tiles)."""
        g = _lib.CGeometry()
        fn = _lib.load().tcs_compute_geometry_ragged if ragged else _lib.load().tcs_compute_geometry
        _lib.check(fn(ctypes.byref(self.to_c()), nx, ny, nz, ctypes.byref(g)))
        return Geometry(tuple(g.grid), tuple(g.elements), tuple(g.threads), g.left_offset, g.right_offset,
                        g.n_points, self.dimension)

    def replace(self, **kw) -> "StencilSpec":
        d = self.__dict__.copy()
        d.update(kw)
        return StencilSpec(**d)


@dataclass(frozen=True)
class Geometry:
    """Grid after truncation to a coarsening multiple and Read/Write padding."""

    grid: tuple            # gridSize (x = padded pitch)
    elements: tuple        # gridElements (interior points per axis)
    threads: tuple         # gridThreads
    left_offset: int
    right_offset: int
    n_points: int
    dimension: int

    @property
    def shape(self) -> tuple:
        """numpy/torch shape of one buffer: (y, x) or (z, y, x)."""
        if self.dimension == 2:
            return (self.grid[1], self.grid[0])
        return (self.grid[2], self.grid[1], self.grid[0])

    @property
    def interior_points(self) -> int:
        e = self.elements
        return e[0] * e[1] * (e[2] if self.dimension == 3 else 1)

    def interior_slices(self, range_: int) -> tuple:
        """Index of the updated interior within a buffer of ``shape``."""
        xs = slice(range_ + self.left_offset, range_ + self.left_offset + self.elements[0])
        ys = slice(range_, range_ + self.elements[1])
        if self.dimension == 2:
            return (ys, xs)
        return (slice(range_, range_ + self.elements[2]), ys, xs)

    def logical_slices(self) -> tuple:
        """Index of the logical grid (without Read/Write padding columns)."""
        xs = slice(self.left_offset, self.grid[0] - self.right_offset)
        if self.dimension == 2:
            return (slice(None), xs)
        return (slice(None), slice(None), xs)
