"""B200-native (sm_100a) thread-coarsened structured-grid stencil engine.

Drop-in for the parameter surface and host interface of MKKnorr/ThreadCoarsenedStencilGenerator:
``StencilSpec`` (generator parameters), ``Stencil`` (one instantiated parameter set, C ABI in
include/tcs.h via ctypes), ``LaunchUpdateGrid`` (the reference's launchUpdateGrid.h) and
``StencilBenchmark`` / ``cli`` (the reference's benchmark host and its TSV report).
"""

from ._lib import CudaErrorInvalidValue, TcsError, UnsupportedLaunch
from .spec import Geometry, StencilSpec
from .stencil import Launch, Plan, Stencil, device_sm_count, precompile, precompile_pipe
from .launch import LaunchUpdateGrid

__all__ = [
    "CudaErrorInvalidValue",
    "Geometry",
    "Launch",
    "LaunchUpdateGrid",
    "Plan",
    "Stencil",
    "StencilSpec",
    "TcsError",
    "UnsupportedLaunch",
    "device_sm_count",
    "precompile",
    "precompile_pipe",
]
