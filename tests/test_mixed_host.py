"""The defect-correction loop of DefectCorrectedSweeps, on the CPU.

The engine's stencils are replaced by stand-ins built on the oracle (FP64 sweep, FP64 defect and
norms, FP32 sweep with a source term, FP64 accumulate), so the loop itself -- the split of n sweeps
into periods, the first correction step taken as a copy of r, the ping-pong of the FP32 fields and
the accumulation -- runs on the host.  After n sweeps the state must equal n FP64 sweeps up to the
FP32 rounding of the corrections.
"""

import numpy as np
import pytest

import oracle as O
from threadcoarsenedstencilgenerator_b200 import mixed
from threadcoarsenedstencilgenerator_b200.spec import StencilSpec

CFG = (2, "Box", "Row", "Variable", 1, 1, 1, 1, "None", 0)


class FakeStencil:
    """Oracle-backed stand-in with the calls the loop makes (CPU torch tensors)."""

    log = []

    def __init__(self, spec):
        self.spec = spec
        self.ospec = O.make_spec(*CFG)
        self.mask = None

    def copy_mask(self, mask):
        self.mask = np.asarray(mask, dtype=np.float64)

    def _interior(self, geom):
        R = self.spec.range
        return slice(R, geom.grid[1] - R), slice(R, geom.grid[0] - R)

    def update_grid(self, geom, src, dst, launch=None, stream=None):
        FakeStencil.log.append(("f64 sweep", self.spec.precision))
        dst.copy_(__import__("torch").from_numpy(O.sweep(self.ospec, src.numpy(), 0, self.mask)))

    def residual(self, geom, x, sx, r, stream=None):
        d = (sx.numpy() - x.numpy())
        r.zero_()
        sl = self._interior(geom)
        r.numpy()[sl] = d[sl].astype(np.float32)
        return float(np.abs(d[sl]).max()), float(np.sqrt((d[sl] ** 2).sum()))

    def update_grid_source(self, geom, a, r, b, launch=None, stream=None):
        FakeStencil.log.append(("f32 sweep", self.spec.precision))
        m32 = None if self.mask is None else self.mask.astype(np.float32)
        out = O.sweep(self.ospec, a.numpy(), 0, m32)
        sl = self._interior(geom)
        out[sl] = out[sl] + r.numpy()[sl]
        b.copy_(__import__("torch").from_numpy(out.astype(np.float32)))

    def accumulate(self, geom, x, e, stream=None):
        sl = self._interior(geom)
        x.numpy()[sl] += e.numpy()[sl].astype(np.float64)

    # the fused sweeps: the same arithmetic as the unfused pairs of calls
    def defect_sweep(self, geom, x, r, launch=None, stream=None):
        FakeStencil.log.append(("f64 sweep", self.spec.precision))
        sx = O.sweep(self.ospec, x.numpy(), 0, self.mask)
        d = sx - x.numpy()
        sl = self._interior(geom)
        r.numpy()[sl] = d[sl].astype(np.float32)
        return float(np.abs(d[sl]).max()), float(np.sqrt((d[sl] ** 2).sum()))

    def update_grid_accumulate(self, geom, a, r, x, launch=None, stream=None):
        import torch

        e = torch.zeros(a.shape, dtype=torch.float32)
        self.update_grid_source(geom, a, r, e)
        self.accumulate(geom, x, e)


@pytest.mark.parametrize("fused", [True, False])
@pytest.mark.parametrize("n, period", [(45, 20), (20, 20), (7, 3), (1, 5), (4, 2)])
def test_defect_correction_loop_tracks_fp64(monkeypatch, n, period, fused):
    import torch

    monkeypatch.setattr(mixed, "Stencil", FakeStencil)
    FakeStencil.log = []
    spec = StencilSpec(dimension=2, neighbourhood="Box", orientation="Row", coefficients="Variable", range=1)
    geom = spec.geometry(40, 30)
    rng = np.random.default_rng(n)
    mask = rng.random(spec.stencil_size)
    mask /= mask.sum()  # a smoothing stencil: the state settles, the corrections shrink
    a = rng.random(geom.shape)
    dc = mixed.DefectCorrectedSweeps(spec, mask=mask, fused=fused)
    x = torch.from_numpy(a.copy())
    x, res = dc.run(geom, x, n, period=period)
    # the fused period gives the unfused period's bits
    FakeStencil.log = []
    other = mixed.DefectCorrectedSweeps(spec, mask=mask, fused=not fused)
    y, _ = other.run(geom, torch.from_numpy(a.copy()), n, period=period)
    assert torch.equal(x, y)
    want = O.sweeps(O.make_spec(*CFG), a, n, 0, mask)
    periods = -(-n // period)
    assert res.fp64_sweeps == periods and res.fp32_sweeps == n and len(res.residual_history) == periods
    # one FP64 sweep per period, k - 1 FP32 steps (the first step is the copy of r)
    assert sum(1 for e in FakeStencil.log if e[0] == "f64 sweep") == periods
    assert sum(1 for e in FakeStencil.log if e[0] == "f32 sweep") == n - periods
    assert np.abs(x.numpy() - want).max() <= 1e-6 * np.abs(want).max()
    # border untouched
    inner = np.zeros(geom.shape, dtype=bool)
    inner[1:-1, 1:-1] = True
    assert np.array_equal(x.numpy()[~inner], a[~inner])
