"""Parameters of the named benchmark workloads, as plain data.

This module imports nothing from the package, so a program can read the workload table without
loading libtcs.so: ``bench.py --impl reference`` times the reference's arithmetic on the host
cores and must not map the engine's library.  ``workloads.py`` builds the engine-side objects
(StencilSpec, Launch) from the same table.

Stencil tuples are (dimension, neighbourhood, orientation, coefficients, range, cx, cy, cz,
alignment, cl_size) -- the generator parameters of cuda/generate2DStencil_cuda.py:15-60 and
cuda/generate3DStencil_cuda.py:15-63.
"""

from __future__ import annotations

import numpy as np

SINGLE = {
    # 2D Box Jacobi r1 (9-point mean), FP64, 4096^2, coarsening 1x1, no alignment, 100 sweeps
    "2d_box_jacobi_r1_4096": {
        "stencil": (2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0),
        "grid": (4096, 4096, 1), "sweeps": 100, "value_range": (0.0, 1.0), "mask_kind": None, "seed": 2024,
        "launch": {"block": (64, 4, 1), "variant": "march"},
        "reference": ((2, 2, 1), (128, 1, 1)),
    },
    # 3D Star Variable r4 (25-point), FP64, 512^3, Read alignment to 16 points, 50 sweeps
    "3d_star_var_r4_512": {
        "stencil": (3, "Star", "Row", "Variable", 4, 1, 2, 2, "Read", 16),
        "grid": (512, 512, 512), "sweeps": 50, "value_range": (0.0, 1.0), "mask_kind": "normal_sum1", "seed": 2024,
        "launch": {"block": (32, 8, 1), "variant": "march"},
        # the reference kernel's best shape over 64 coarsening triples x 46 blocks (oracle/ref_sweep.py)
        "reference": ((3, 4, 3), (32, 2, 2)),
    },
    # 2D Box Variable r6 (169-point), FP64, 16384x8192, mask N(0,1)/169, values U[-1,1], 200 sweeps
    "2d_box_var_r6_16384x8192": {
        "stencil": (2, "Box", "Row", "Variable", 6, 2, 4, 1, "None", 0),
        "grid": (16384, 8192, 1), "sweeps": 200, "value_range": (-1.0, 1.0), "mask_kind": "normal_over_S",
        "seed": 2024, "launch": {"block": (32, 4, 1), "variant": "march"},
        "reference": ((2, 4, 1), (32, 4, 1)),
    },
}

BATCH = {
    # 64 independent 3D Star Jacobi r2 grids, sides log-uniform in [64, 256] (multiples of the
    # coarsening 2x2x2), values U[0,1), 50 sweeps per run, FP64 and FP32
    "batch_3d_star_jacobi_r2_64": {
        "stencil": (3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0),
        "n_grids": 64, "side_range": (64, 256), "multiple": 2, "sweeps": 50, "seed": 2024,
    },
}

DEFAULT = "3d_star_var_r4_512"


def stencil_size(stencil: tuple) -> int:
    """Points of the neighbourhood (cuda/generate2DStencil_cuda.py:63-67,
    cuda/generate3DStencil_cuda.py:66-70)."""
    d, sh, r = stencil[0], stencil[1], stencil[4]
    w = 2 * r + 1
    if sh == "Box":
        return w ** d
    return 2 * d * r + 1


def make_input(seed: int, value_range: tuple, shape: tuple, dtype=np.float64) -> np.ndarray:
    """Seeded input grid: numpy default_rng(seed) uniform draws, scaled to value_range."""
    rng = np.random.default_rng(seed)
    lo, hi = value_range
    a = rng.random(shape, dtype=np.float64 if dtype == np.float64 else np.float32)
    if (lo, hi) != (0.0, 1.0):
        a = a * (hi - lo) + lo
    return a.astype(dtype, copy=False)


def make_mask(seed: int, mask_kind: str | None, stencil: tuple) -> np.ndarray | None:
    """Seeded Variable mask: N(0,1) from default_rng(seed + 1), normalised to sum 1
    ("normal_sum1") or divided by the stencil size ("normal_over_S")."""
    if mask_kind is None or stencil[3] == "Jacobi":
        return None
    S = stencil_size(stencil)
    m = np.random.default_rng(seed + 1).standard_normal(S)
    if mask_kind == "normal_sum1":
        return m / m.sum()
    return m / S


def batch_sides(n_grids: int, side_range: tuple, multiple: int, seed: int) -> list:
    """Grid extents (nx, ny, nz) per grid, drawn per axis log-uniform from default_rng(seed)."""
    rng = np.random.default_rng(seed)
    lo, hi = side_range
    u = rng.uniform(np.log(lo), np.log(hi), size=(n_grids, 3))
    s = np.rint(np.exp(u) / multiple).astype(np.int64) * multiple
    s = np.clip(s, lo, hi)
    return [tuple(int(v) for v in row) for row in s]


def batch_inputs(seed: int, shapes: list, dtype=np.float64) -> list:
    """Values uniform [0, 1) per grid (one stream of draws from default_rng(seed + 1), grid after
    grid)."""
    rng = np.random.default_rng(seed + 1)
    return [rng.random(s, dtype=np.float64).astype(dtype, copy=False) for s in shapes]
