"""Build and run the host build of the engine's per-thread arithmetic (see tile_host.cpp)."""

from __future__ import annotations

import ctypes
import hashlib
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
CSRC = ROOT / "threadcoarsenedstencilgenerator_b200" / "csrc"
OUT = ROOT / "_build" / "host_tile"

_SH = {"Box": 0, "Star": 1}
_OR = {"Row": 0, "Column": 1}
_CO = {"Jacobi": 0, "Variable": 1}


def build(cfg, precision="f64", source="tile_host.cpp") -> ctypes.CDLL:
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    macros = {
        "TCS_T": "double" if precision == "f64" else "float",
        "TCS_DIM": d, "TCS_SHAPE": _SH[sh], "TCS_ORIENT": _OR[o], "TCS_COEFF": _CO[c], "TCS_R": r,
        "TCS_CX": cx, "TCS_CY": cy, "TCS_CZ": cz if d == 3 else 1,
    }
    if precision == "f32c":  # FP32 grids, compensated accumulation
        macros["TCS_COMP"] = 1
    src = (HERE / source).read_bytes() + (HERE / "host_cuda_shim.h").read_bytes() + (CSRC / "tcs_tile.cuh").read_bytes()
    tag = hashlib.sha1(src + repr(sorted(macros.items())).encode()).hexdigest()[:16]
    OUT.mkdir(parents=True, exist_ok=True)
    so = OUT / ("tile_%s.so" % tag)
    if not so.exists():
        cmd = ["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-Wno-unknown-pragmas", "-shared", "-fPIC",
               "-I", str(CSRC), "-I", str(HERE)] + ["-D%s=%s" % kv for kv in macros.items()] + [str(HERE / source),
                                                                              "-o", str(so) + ".tmp"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(proc.stderr[-3000:])
        Path(str(so) + ".tmp").rename(so)
    return ctypes.CDLL(str(so))


def sweeps(cfg, a: np.ndarray, grid, left_offset, right_offset, n: int, mask=None, precision="f64"):
    lib = build(cfg, precision)
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    x = np.ascontiguousarray(a).copy()
    y = x.copy()
    m = np.ascontiguousarray(np.zeros(1) if mask is None else np.asarray(mask, dtype=np.float64))
    u3 = ctypes.c_uint * 3
    for _ in range(n):
        lib.tile_sweep(u3(*grid), ctypes.c_uint(left_offset), ctypes.c_uint(right_offset),
                       ctypes.c_int(0 if al == "None" else 1), x.ctypes.data_as(ctypes.c_void_p),
                       y.ctypes.data_as(ctypes.c_void_p), m.ctypes.data_as(ctypes.c_void_p))
        x, y = y, x
    return x


def pipe_sweeps(cfg, a: np.ndarray, grid, left_offset, right_offset, n: int, mask=None, precision="f64",
                piece: int = 1 << 30, unroll: int = 0):
    """n sweeps through the host build of the pipelined sweep (pieces of `piece` planes)."""
    lib = build(cfg, precision, "pipe_host.cpp")
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    unroll = unroll or 2 * r + 1
    x = np.ascontiguousarray(a).copy()
    y = x.copy()
    m = np.ascontiguousarray(np.zeros(1) if mask is None else np.asarray(mask, dtype=np.float64))
    u3 = ctypes.c_uint * 3
    for _ in range(n):
        lib.pipe_sweep(u3(*grid), ctypes.c_uint(left_offset), ctypes.c_uint(right_offset),
                       ctypes.c_int(0 if al == "None" else 1), x.ctypes.data_as(ctypes.c_void_p),
                       y.ctypes.data_as(ctypes.c_void_p), m.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(piece),
                       ctypes.c_uint(unroll))
        x, y = y, x
    return x


def pipe_ring_sweeps(cfg, a: np.ndarray, grid, left_offset, right_offset, n: int, mask=None, precision="f64",
                     piece: int = 1 << 30):
    """n sweeps through the host build of the ring form of the pipelined sweep (3D Star, Row)."""
    lib = build(cfg, precision, "pipe_host.cpp")
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    x = np.ascontiguousarray(a).copy()
    y = x.copy()
    m = np.ascontiguousarray(np.zeros(1) if mask is None else np.asarray(mask, dtype=np.float64))
    u3 = ctypes.c_uint * 3
    for _ in range(n):
        rc = lib.pipe_sweep_ring(u3(*grid), ctypes.c_uint(left_offset), ctypes.c_uint(right_offset),
                                 ctypes.c_int(0 if al == "None" else 1), x.ctypes.data_as(ctypes.c_void_p),
                                 y.ctypes.data_as(ctypes.c_void_p), m.ctypes.data_as(ctypes.c_void_p),
                                 ctypes.c_uint(piece))
        assert rc == 0
        x, y = y, x
    return x


def tb3_passes(cfg, a: np.ndarray, grid, left_offset, right_offset, n: int, mask=None, precision="f64",
               block=(8, 8), piece: int = 1 << 30, unroll: int = 2):
    """n passes (2n sweeps) through the host build of the two-sweep kernel's control flow,
    compiled with the kernel's own thread tile (3D: 2 x 2 for even ranges, 1 x 1 for odd ones;
    2D: 2 x 1, and block[1] is ignored)."""
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    C = 2 if (r % 2 == 0 or d == 2) else 1
    lib = build((d, sh, o, c, r, C, C if d == 3 else 1, 1, al, cl), precision, "tb3_host.cpp")
    x = np.ascontiguousarray(a).copy()
    y = x.copy()
    m = np.ascontiguousarray(np.zeros(1) if mask is None else np.asarray(mask, dtype=np.float64))
    u3 = ctypes.c_uint * 3
    for _ in range(n):
        rc = lib.tb3_pass(u3(*grid), ctypes.c_uint(left_offset), ctypes.c_uint(right_offset),
                          ctypes.c_int(0 if al == "None" else 1), x.ctypes.data_as(ctypes.c_void_p),
                          y.ctypes.data_as(ctypes.c_void_p), m.ctypes.data_as(ctypes.c_void_p),
                          ctypes.c_uint(block[0]), ctypes.c_uint(block[1]), ctypes.c_uint(piece),
                          ctypes.c_uint(unroll))
        assert rc == 0
        x, y = y, x
    return x
