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

from . import workload_params as P
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
        return P.make_input(self.seed, self.value_range, geom.shape, dtype)

    def make_mask(self) -> np.ndarray | None:
        return P.make_mask(self.seed, self.mask_kind, _stencil_tuple(self.spec))

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
                              chunk=int(t.get("chunk", 0)), tmem=bool(t.get("tmem", False)),
                              lockstep=bool(t.get("lockstep", False)))
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


def _spec_of(t: tuple) -> StencilSpec:
    d, sh, o, c, r, cx, cy, cz, al, cl = t
    return StencilSpec(dimension=d, neighbourhood=sh, orientation=o, coefficients=c, range=r, cx=cx, cy=cy, cz=cz,
                       alignment=al, cl_size=cl)


def _stencil_tuple(s: StencilSpec) -> tuple:
    return (s.dimension, s.neighbourhood, s.orientation, s.coefficients, s.range, s.cx, s.cy, s.cz, s.alignment,
            s.cl_size)


WORKLOADS = {
    name: Workload(name=name, spec=_spec_of(p["stencil"]), grid=tuple(p["grid"]), sweeps=p["sweeps"],
                   value_range=tuple(p["value_range"]), mask_kind=p["mask_kind"], seed=p["seed"],
                   launch=Launch(block=tuple(p["launch"]["block"]), variant=p["launch"]["variant"]),
                   reference=tuple(p["reference"]))
    for name, p in P.SINGLE.items()
}

DEFAULT_WORKLOAD = P.DEFAULT


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
        return P.batch_sides(self.n_grids, self.side_range, self.multiple, self.seed)

    def geometries(self, spec: StencilSpec | None = None) -> list:
        spec = spec or self.spec
        return [spec.geometry(*sd) for sd in self.sides()]

    def make_inputs(self, geoms, dtype=np.float64) -> list:
        """Values uniform [0, 1) per grid (one stream of draws, grid after grid)."""
        return P.batch_inputs(self.seed, [g.shape for g in geoms], dtype)

    def tuned_launch(self, precision: str = "f64") -> Launch:
        """Launch chosen by the autotuner for this batch (per precision), else the default."""
        if TUNED_PATH.exists():
            t = json.loads(TUNED_PATH.read_text()).get(self.name + ("" if precision == "f64" else "_" + precision))
            if t:
                return Launch(block=tuple(t["block"]), variant="pipe", segments=int(t.get("segments", 0)),
                              depth=int(t.get("depth", 0)), chunk=int(t.get("chunk", 0)))
        return self.launch


BATCH_WORKLOADS = {
    name: BatchWorkload(name=name, spec=_spec_of(p["stencil"]), n_grids=p["n_grids"],
                        side_range=tuple(p["side_range"]), multiple=p["multiple"], sweeps=p["sweeps"], seed=p["seed"])
    for name, p in P.BATCH.items()
}
