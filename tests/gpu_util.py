"""Helpers of the GPU tests: run the engine and the reference's own kernels on the same inputs."""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from oracle import ref_configs

ROOT = Path(__file__).resolve().parents[1]


def spec_of(cfg, precision="f64"):
    import threadcoarsenedstencilgenerator_b200 as tcs

    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    return tcs.StencilSpec(dimension=d, neighbourhood=sh, orientation=o, coefficients=c, range=r, cx=cx, cy=cy,
                           cz=cz, alignment=al, cl_size=cl, precision=precision)


def engine_sweeps(stencil, geom, a: np.ndarray, n: int, launch, mask=None, sentinel_padding=True):
    """Upload a into both buffers (fixed border), run n sweeps, return (result, other buffer)."""
    import torch

    dt = torch.float64 if a.dtype == np.float64 else torch.float32
    host = torch.from_numpy(np.ascontiguousarray(a))
    if sentinel_padding:
        host = host.clone()
        ls = geom.logical_slices()
        pad = torch.ones(host.shape, dtype=torch.bool)
        pad[ls] = False
        host[pad] = float("nan")
    x = host.to("cuda", dtype=dt)
    y = x.clone()
    if mask is not None:
        stencil.copy_mask(mask)
    res = stencil.sweeps(geom, x, y, n, launch)
    torch.cuda.synchronize()
    other = y if res is x else x
    return res.cpu().numpy(), other.cpu().numpy(), host.numpy()


def ref_lib_path(cfg) -> Path:
    return ROOT / "oracle" / "_ref" / ref_configs.key(cfg) / "libref.so"


def reference_sweeps(cfg, geom_grid, threads, right_offset, a: np.ndarray, n: int, mask=None, block=None):
    """n sweeps of the reference's own generated kernel (sm_100a build) through benchmarkUpdateGrid."""
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    lib = ctypes.CDLL(str(ref_lib_path(cfg)))
    u3 = ctypes.c_uint * 3
    block = block or ((8, 4, 2) if d == 3 else (8, 4, 1))
    gb = tuple(max(1, -(-threads[i] // block[i])) for i in range(3))
    a = np.ascontiguousarray(a, dtype=np.float64)
    out = np.empty_like(a)
    m = np.zeros(1) if mask is None else np.ascontiguousarray(mask, dtype=np.float64)
    rc = lib.ref_sweeps(c.encode(), sh.encode(), ctypes.c_uint(r), ctypes.c_uint(d), al.encode(), u3(*geom_grid),
                        u3(*block), u3(*gb), ctypes.c_uint(right_offset), m.ctypes.data_as(ctypes.c_void_p),
                        ctypes.c_uint(0 if mask is None else m.size), a.ctypes.data_as(ctypes.c_void_p),
                        out.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(n))
    assert rc == 0, "reference run failed (%d)" % rc
    return out
