"""FP32 sweeps with FP64 defect correction (mixed-precision sweep of a linear stencil).

One FP64 sweep is x -> S(x) = A x + b, with A the stencil on the interior and b the contribution
of the fixed border.  Every ``period`` sweeps the engine
  1. computes the defect r = S(x) - x in FP64 on the GPU (one FP64 sweep plus ``tcs_residual``,
     which also returns the global residual norms in FP64),
  2. runs ``period`` FP32 sweeps of the correction recurrence e <- A e + r from e = 0 (zero border;
     the source term r is added in the sweep epilogue, ``tcs_update_grid_source``).  The first
     step gives e = r exactly (A 0 = 0), so it is a copy of r instead of a sweep,
  3. accumulates x += e in FP64 (``tcs_accumulate``).
In exact arithmetic e after k steps equals sum_{i<k} A^i r, so x + e is exactly the FP64 state k
sweeps later; rounding enters only through the FP32 correction, whose size is the change of the
state over the period, so the result tracks the FP64 iteration to far better than FP32 precision
once the iteration settles.

By default the period runs fused (pipelined kernel, grids of whole coarsening tiles): step 1 is one
FP64 sweep whose epilogue writes r and the norms without storing S(x) (``tcs_defect_sweep``), the
first FP32 sweep reads r directly instead of a copy of it, and the last FP32 sweep adds its result
into x in its epilogue (``tcs_update_grid_accumulate``).  Every value is bit-identical to the
unfused sequence; only the order in which the 2-norm is summed differs.  The FP32 sweeps are the engine's ordinary single-precision kernels,
or, with ``tensor_cores=True`` (2D Box stencils), the tcgen05 banded contraction with BF16 high and
low parts and FP32 accumulation (``tcs_tc_update_grid``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

from .spec import Geometry, StencilSpec
from .stencil import Launch, Stencil


@dataclass
class MixedResult:
    sweeps: int
    fp64_sweeps: int
    fp32_sweeps: int  # steps of the FP32 recurrence (the first of every period is a copy of r)
    residual_history: list = field(default_factory=list)  # (max |r|, ||r||_2) per period


class DefectCorrectedSweeps:
    """Run n sweeps of ``spec`` (FP64 semantics) as FP32 sweeps with periodic FP64 defect correction."""

    def __init__(self, spec: StencilSpec, launch64: Launch | None = None, launch32: Launch | None = None,
                 mask=None, tensor_cores: bool = False, coarsening32: tuple | None = None, fused: bool = True):
        """``launch32`` and ``coarsening32`` give the FP32 sweeps a launch shape of their own (FP32
        keeps twice the values per register and runs at twice the FP64 rate, so its best shape
        differs); the per-point arithmetic does not depend on either."""
        if spec.precision != "f64":
            spec = spec.replace(precision="f64")
        self.spec64 = spec
        self.spec32 = spec.replace(precision="f32")
        if coarsening32 is not None:
            c = tuple(coarsening32) + (1,) * (3 - len(coarsening32))
            self.spec32 = self.spec32.replace(cx=c[0], cy=c[1], cz=c[2] if spec.dimension == 3 else 1)
        self.s64 = Stencil(self.spec64)
        self.s32 = Stencil(self.spec32)
        if mask is not None:
            self.s64.copy_mask(mask)
            self.s32.copy_mask(mask)
        self.launch64 = launch64 or Launch()
        self.launch32 = launch32 or self.launch64
        self.tensor_cores = tensor_cores
        self.fused = fused
        self._accumulate_ok = True

    def run(self, geom: Geometry, x, n: int, period: int = 20, stream=None, work=None) -> tuple:
        """Advance the FP64 state ``x`` (torch float64 tensor of geom.shape) by n sweeps in place.

        ``work`` may hold preallocated buffers {"sx": f64, "r": f32, "e0": f32, "e1": f32}; they
        are created with torch otherwise.  Returns (x, MixedResult)."""
        import torch

        if work is None:
            work = {"sx": x.clone(), "r": torch.zeros(geom.shape, dtype=torch.float32, device=x.device),
                    "e0": torch.zeros(geom.shape, dtype=torch.float32, device=x.device),
                    "e1": torch.zeros(geom.shape, dtype=torch.float32, device=x.device)}
        sx, r, e0, e1 = work["sx"], work["r"], work["e0"], work["e1"]
        sx.copy_(x)  # the border of S(x) is x's border
        r.zero_()    # the correction fields keep a zero border: r's is copied into e0 each period
        e0.zero_()
        e1.zero_()
        res = MixedResult(n, 0, 0)
        done = 0
        while done < n:
            k = min(period, n - done)
            if self.fused and self._fused_period(geom, x, k, r, e0, e1, res, stream):
                done += k
                continue
            self.s64.update_grid(geom, x, sx, self.launch64, stream)
            norms = self.s64.residual(geom, x, sx, r, stream)
            res.residual_history.append(norms)
            res.fp64_sweeps += 1
            e0.copy_(r)  # e after the first step: A 0 + r = r
            a, b = e0, e1
            for _ in range(k - 1):
                if self.tensor_cores:
                    self.s32.tc_update_grid(geom, a, b, source=r, stream=stream)
                else:
                    self.s32.update_grid_source(geom, a, r, b, self.launch32, stream)
                a, b = b, a
            res.fp32_sweeps += k
            self.s64.accumulate(geom, x, a, stream)
            done += k
        return x, res

    def _fused_period(self, geom: Geometry, x, k: int, r, e0, e1, res: MixedResult, stream) -> bool:
        """One period through the fused sweeps; False (nothing done) when the launch cannot run
        them, which turns fusion off for this object."""
        from ._lib import UnsupportedLaunch

        try:
            norms = self.s64.defect_sweep(geom, x, r, self.launch64, stream)
        except UnsupportedLaunch:
            self.fused = False
            return False
        res.residual_history.append(norms)
        res.fp64_sweeps += 1
        a, bufs = r, (e0, e1)  # the recurrence starts from e = r: read r itself
        for i in range(k - 1):
            last = i == k - 2
            b = bufs[i % 2]
            if self.tensor_cores:
                self.s32.tc_update_grid(geom, a, b, source=r, stream=stream)
            elif last and self._accumulate_ok:
                try:
                    self.s32.update_grid_accumulate(geom, a, r, x, self.launch32, stream)
                    a = None
                    break
                except UnsupportedLaunch:
                    self._accumulate_ok = False
                    self.s32.update_grid_source(geom, a, r, b, self.launch32, stream)
            else:
                self.s32.update_grid_source(geom, a, r, b, self.launch32, stream)
            a = b
        if a is not None:
            self.s64.accumulate(geom, x, a, stream)
        res.fp32_sweeps += k
        return True
