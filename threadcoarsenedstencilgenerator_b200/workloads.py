"""Named benchmark workloads: the stencil configurations the engine is measured on.

Each workload fixes a parameter set, a grid, the number of sweeps of one run, how the seeded
synthetic input and mask are drawn, and the launch the engine uses for it (the autotuner's choice,
see ``tuned.json``).  Inputs are numpy ``default_rng(seed)`` draws, so the oracle and the engine
see identical data.
"""

from __future__ import annotations

import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .spec import StencilSpec
from .stencil import Launch

TUNED_PATH = Path(__file__).resolve().parent / "tuned.json"


@dataclass(frozen=True)
class Workload:
    name: str
    spec: StencilSpec
    grid: tuple                  # raw grid size (nx, ny, nz) before truncation/padding
    sweeps: int                  # sweeps of one run
    value_range: tuple = (0.0, 1.0)
    mask_kind: str | None = None  # "normal_sum1" | "normal_over_S" | None
    seed: int = 2024
    launch: Launch = field(default_factory=Launch)
    reference: tuple = ()        # (coarsening, block) of the reference kernel timed beside it

    def geometry(self):
        return self.spec.geometry(*self.grid)

    def make_input(self, geom, dtype=np.float64) -> np.ndarray:
        rng = np.random.default_rng(self.seed)
        lo, hi = self.value_range
        a = rng.random(geom.shape, dtype=np.float64 if dtype == np.float64 else np.float32)
        if (lo, hi) != (0.0, 1.0):
            a = a * (hi - lo) + lo
        return a.astype(dtype, copy=False)

    def make_mask(self) -> np.ndarray | None:
        if self.mask_kind is None or self.spec.coefficients == "Jacobi":
            return None
        S = self.spec.stencil_size
        rng = np.random.default_rng(self.seed + 1)
        m = rng.standard_normal(S)
        if self.mask_kind == "normal_sum1":
            return m / m.sum()
        return m / S

    def _tuned(self, precision: str):
        if not TUNED_PATH.exists():
            return None
        d = json.loads(TUNED_PATH.read_text())
        return d.get(self.name + "_" + precision) if precision != "f64" and self.name + "_" + precision in d \
            else d.get(self.name)

    def tuned_launch(self, precision: str = "f64") -> Launch:
        """Launch chosen by the autotuner for this workload and precision (an entry
        ``<name>_<precision>`` when the precision has its own, else the FP64 one; falls back to the
        built-in default)."""
        if TUNED_PATH.exists():
            t = self._tuned(precision)
            if t:
                return Launch(block=tuple(t["block"]), variant=t.get("variant", "auto"),
                              segments=int(t.get("segments", 0)), depth=int(t.get("depth", 0)),
                              chunk=int(t.get("chunk", 0)))
        return self.launch

    def tuned_spec(self, precision: str = "f64") -> StencilSpec:
        """Parameter set with the coarsening chosen by the autotuner for this precision (same
        stencil arithmetic; the precision of the result is the workload's own)."""
        if TUNED_PATH.exists():
            t = self._tuned(precision)
            if t and "coarsening" in t:
                c = t["coarsening"]
                return self.spec.replace(cx=c[0], cy=c[1], cz=c[2] if self.spec.dimension == 3 else 1)
        return self.spec


WORKLOADS = {
    # 2D Box Jacobi r1 (9-point mean), FP64, 4096^2, coarsening 1x1, no alignment, 100 sweeps
    "2d_box_jacobi_r1_4096": Workload(
        name="2d_box_jacobi_r1_4096",
        spec=StencilSpec(dimension=2, neighbourhood="Box", orientation="Row", coefficients="Jacobi", range=1),
        grid=(4096, 4096, 1), sweeps=100, launch=Launch(block=(64, 4, 1), variant="march"),
        reference=((2, 2, 1), (128, 1, 1))),
    # 3D Star Variable r4 (25-point), FP64, 512^3, Read alignment to 16 points, 50 sweeps
    "3d_star_var_r4_512": Workload(
        name="3d_star_var_r4_512",
        spec=StencilSpec(dimension=3, neighbourhood="Star", orientation="Row", coefficients="Variable", range=4,
                         cx=1, cy=2, cz=2, alignment="Read", cl_size=16),
        grid=(512, 512, 512), sweeps=50, mask_kind="normal_sum1", launch=Launch(block=(32, 8, 1), variant="march"),
        reference=((1, 4, 2), (128, 2, 1))),
    # 2D Box Variable r6 (169-point), FP64, 16384x8192, mask N(0,1)/169, values U[-1,1], 200 sweeps
    "2d_box_var_r6_16384x8192": Workload(
        name="2d_box_var_r6_16384x8192",
        spec=StencilSpec(dimension=2, neighbourhood="Box", orientation="Row", coefficients="Variable", range=6,
                         cx=2, cy=4),
        grid=(16384, 8192, 1), sweeps=200, value_range=(-1.0, 1.0), mask_kind="normal_over_S",
        launch=Launch(block=(32, 4, 1), variant="march"), reference=((2, 4, 1), (32, 4, 1))),
}

DEFAULT_WORKLOAD = "3d_star_var_r4_512"


@dataclass(frozen=True)
class BatchWorkload:
    """Many independent grids of one parameter set with seeded uneven extents."""

    name: str
    spec: StencilSpec
    n_grids: int
    side_range: tuple            # each side log-uniform in [lo, hi]
    multiple: int                # sides rounded to a multiple of this (the coarsening)
    sweeps: int
    seed: int = 2024
    launch: Launch = field(default_factory=lambda: Launch(block=(32, 4, 1), variant="pipe"))

    def sides(self) -> list:
        """Grid extents (nx, ny, nz) per grid, drawn per axis from default_rng(seed)."""
        rng = np.random.default_rng(self.seed)
        lo, hi = self.side_range
        u = rng.uniform(np.log(lo), np.log(hi), size=(self.n_grids, 3))
        s = np.rint(np.exp(u) / self.multiple).astype(np.int64) * self.multiple
        s = np.clip(s, lo, hi)
        return [tuple(int(v) for v in row) for row in s]

    def geometries(self, spec: StencilSpec | None = None) -> list:
        spec = spec or self.spec
        return [spec.geometry(*sd) for sd in self.sides()]

    def make_inputs(self, geoms, dtype=np.float64) -> list:
        """Values uniform [0, 1) per grid (one stream of draws, grid after grid)."""
        rng = np.random.default_rng(self.seed + 1)
        return [rng.random(g.shape, dtype=np.float64).astype(dtype, copy=False) for g in geoms]

    def tuned_launch(self, precision: str = "f64") -> Launch:
        """Launch chosen by the autotuner for this batch (per precision), else the default."""
        if TUNED_PATH.exists():
            t = json.loads(TUNED_PATH.read_text()).get(self.name + ("" if precision == "f64" else "_" + precision))
            if t:
                return Launch(block=tuple(t["block"]), variant="pipe", segments=int(t.get("segments", 0)),
                              depth=int(t.get("depth", 0)), chunk=int(t.get("chunk", 0)))
        return self.launch


BATCH_WORKLOADS = {
    # 64 independent 3D Star Jacobi r2 grids, sides log-uniform in [64, 256] (multiples of the
    # coarsening 2x2x2), values U[0,1), 50 sweeps per run, FP64 and FP32
    "batch_3d_star_jacobi_r2_64": BatchWorkload(
        name="batch_3d_star_jacobi_r2_64",
        spec=StencilSpec(dimension=3, neighbourhood="Star", orientation="Row", coefficients="Jacobi", range=2,
                         cx=2, cy=2, cz=2),
        n_grids=64, side_range=(64, 256), multiple=2, sweeps=50),
}
