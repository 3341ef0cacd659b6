"""Mixed-precision pieces on the GPU: source-term sweeps, FP64 defect and norms, accumulation,
error statistics, and the defect-corrected FP32 iteration against the FP64 oracle.

Tolerances: source sweeps, defect values and accumulation are exact (0 ulp); norms and error
statistics are FP64 reductions in a different order than numpy's (relative 1e-12); the
defect-corrected iteration must match the FP64 oracle to max and RMS relative error <= 1e-6
(relative to max |x| and ||x||_2 of the FP64 result), the bound the FP32 forms are held to."""

import numpy as np
import pytest

import gpu_util as G
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tcs():
    import threadcoarsenedstencilgenerator_b200 as t

    return t


SOURCE_CASES = [
    ((2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0), (32, 1, 1), "pipe"),
    ((2, "Box", "Row", "Variable", 2, 2, 2, 1, "Read", 16), (32, 4, 1), "march"),
    ((3, "Star", "Row", "Variable", 2, 2, 2, 1, "None", 0), (16, 2, 1), "pipe"),
    ((3, "Box", "Column", "Jacobi", 1, 1, 1, 1, "Write", 8), (32, 4, 1), "direct"),
]


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("case", SOURCE_CASES, ids=lambda c: "%s_%s" % (c[2], c[0][1]))
def test_source_sweep_is_stencil_plus_source(tcs, case, precision):
    import torch

    cfg, block, variant = case
    spec = G.spec_of(cfg, precision)
    st = tcs.Stencil(spec)
    geom = spec.geometry(70, 41, 23)
    rng = np.random.default_rng(3)
    dt = np.float64 if precision == "f64" else np.float32
    a = rng.random(geom.shape).astype(dt)
    src = rng.standard_normal(geom.shape).astype(dt)
    mask = rng.standard_normal(spec.stencil_size) if cfg[3] == "Variable" else None
    if mask is not None:
        st.copy_mask(mask)
    want = O.sweep(O.make_spec(*cfg), a, geom.right_offset, mask)
    sl = geom.interior_slices(cfg[4])
    want[sl] = want[sl] + src[sl]
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    s = torch.from_numpy(src).cuda()
    st.update_grid_source(geom, x, s, y, tcs.Launch(block=block, variant=variant))
    assert np.array_equal(y.cpu().numpy(), want)


def test_residual_accumulate_compare(tcs):
    import torch

    cfg = (3, "Star", "Row", "Variable", 2, 1, 1, 1, "Read", 16)
    spec = G.spec_of(cfg)
    st = tcs.Stencil(spec)
    geom = spec.geometry(60, 33, 27)
    rng = np.random.default_rng(9)
    x = rng.random(geom.shape)
    sx = x + 1e-3 * rng.standard_normal(geom.shape)
    sl = geom.interior_slices(2)
    xd, sxd = torch.from_numpy(x).cuda(), torch.from_numpy(sx).cuda()
    r = torch.zeros(geom.shape, dtype=torch.float32, device="cuda")
    mx, l2 = st.residual(geom, xd, sxd, r)
    d = (sx - x)[sl]
    assert np.array_equal(r.cpu().numpy()[sl], d.astype(np.float32))
    assert np.all(r.cpu().numpy()[np.ones(geom.shape, bool) & ~_mask(geom.shape, sl)] == 0)
    assert mx == np.abs(d).max() and abs(l2 - np.sqrt((d * d).sum())) <= 1e-12 * l2
    e = rng.standard_normal(geom.shape).astype(np.float32)
    ed = torch.from_numpy(e).cuda()
    st.accumulate(geom, xd, ed)
    want = x.copy()
    want[sl] = want[sl] + e[sl].astype(np.float64)
    assert np.array_equal(xd.cpu().numpy(), want)
    stats = st.compare(geom, ed, xd, "f32")
    diff = e[sl].astype(np.float64) - want[sl]
    assert stats["max_abs"] == np.abs(diff).max()
    assert abs(stats["l2"] - np.sqrt((diff * diff).sum())) <= 1e-12 * stats["l2"]
    assert stats["max_ref"] == np.abs(want[sl]).max()


def _mask(shape, sl):
    m = np.zeros(shape, bool)
    m[sl] = True
    return m


@pytest.mark.parametrize("cfg,n,period", [
    ((2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0), 60, 20),
    ((3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16), 40, 10),
])
def test_defect_corrected_fp32_tracks_fp64(tcs, cfg, n, period):
    import torch

    from threadcoarsenedstencilgenerator_b200.mixed import DefectCorrectedSweeps

    spec = G.spec_of(cfg)
    geom = spec.geometry(300, 200, 1) if cfg[0] == 2 else spec.geometry(64, 48, 40)
    rng = np.random.default_rng(21)
    a = rng.random(geom.shape) * 2.0 - 1.0
    m = rng.standard_normal(spec.stencil_size)
    mask = m / spec.stencil_size if cfg[1] == "Box" else m / m.sum()
    want = O.sweeps(O.make_spec(*cfg), a, n, geom.right_offset, mask, cpu_threads=0)
    block = (32, 1, 1) if cfg[0] == 2 else (16, 2, 1)
    dc = DefectCorrectedSweeps(spec, tcs.Launch(block=block, variant="pipe"), mask=mask)
    x = torch.from_numpy(a).cuda()
    x, res = dc.run(geom, x, n, period)
    assert res.fp64_sweeps == -(-n // period) and res.fp32_sweeps == n
    b = torch.from_numpy(want).cuda()
    stats = dc.s64.compare(geom, x, b, "f64")
    assert stats["max_rel"] <= 1e-6 and stats["rms_rel"] <= 1e-6, stats
    # the plain FP32 iteration, for contrast, is reported but only bounded loosely
    x32 = torch.from_numpy(a.astype(np.float32)).cuda()
    y32 = x32.clone()
    res32 = dc.s32.sweeps(geom, x32, y32, n, tcs.Launch(block=block, variant="pipe"))
    s32 = dc.s64.compare(geom, res32, b, "f32")
    assert s32["max_rel"] < 1e-3
    assert dc.s64.device_status() == 0 and dc.s32.device_status() == 0


FUSED_CASES = [
    ((2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0), (32, 1, 1), (300, 90, 1)),
    ((3, "Star", "Row", "Variable", 2, 2, 2, 1, "Read", 16), (16, 4, 1), (70, 42, 30)),
    ((3, "Box", "Row", "Jacobi", 1, 2, 1, 1, "None", 0), (32, 2, 1), (66, 20, 19)),
]


@pytest.mark.parametrize("case", FUSED_CASES, ids=lambda c: "%dD_%s_%s_r%d" % (c[0][0], c[0][1], c[0][3], c[0][4]))
def test_fused_defect_and_accumulate_sweeps(tcs, case):
    """tcs_defect_sweep == one FP64 sweep + tcs_residual (r bit for bit, max norm exact, 2-norm to
    1e-12); tcs_update_grid_accumulate == tcs_update_grid_source + tcs_accumulate (bit for bit)."""
    import torch

    cfg, block, sides = case
    s64 = tcs.Stencil(G.spec_of(cfg, "f64"))
    s32 = tcs.Stencil(G.spec_of(cfg, "f32"))
    geom = s64.spec.geometry(*sides[:cfg[0]])
    rng = np.random.default_rng(17)
    mask = rng.standard_normal(s64.spec.stencil_size) / s64.spec.stencil_size if cfg[3] == "Variable" else None
    if mask is not None:
        s64.copy_mask(mask)
        s32.copy_mask(mask)
    launch = tcs.Launch(block=block, variant="pipe")
    x = torch.from_numpy(rng.uniform(-1, 1, geom.shape)).cuda()
    sx = x.clone()
    r_ref = torch.zeros(geom.shape, dtype=torch.float32, device="cuda")
    r = torch.full(geom.shape, 0.0, dtype=torch.float32, device="cuda")
    s64.update_grid(geom, x, sx, launch)
    n_ref = s64.residual(geom, x, sx, r_ref)
    n_fused = s64.defect_sweep(geom, x, r, launch)
    torch.cuda.synchronize()
    assert torch.equal(r, r_ref)
    assert n_fused[0] == n_ref[0]
    assert abs(n_fused[1] - n_ref[1]) <= 1e-12 * n_ref[1]
    # accumulate: x2 += S(e) + r  against  e1 = S(e) + r; x1 += e1
    e = torch.from_numpy(rng.standard_normal(geom.shape).astype(np.float32) * 1e-3).cuda()
    sl = geom.interior_slices(cfg[4])
    outside = torch.ones(geom.shape, dtype=torch.bool)
    outside[sl] = False
    e[outside.cuda()] = 0
    x1, x2 = x.clone(), x.clone()
    e1 = torch.zeros_like(e)
    s32.update_grid_source(geom, e, r, e1, launch)
    s64.accumulate(geom, x1, e1)
    s32.update_grid_accumulate(geom, e, r, x2, launch)
    # the same buffer as input and source (the first correction step of a period of two)
    x3, x4 = x.clone(), x.clone()
    e2 = torch.zeros_like(e)
    s32.update_grid_source(geom, r, r, e2, launch)
    s64.accumulate(geom, x3, e2)
    s32.update_grid_accumulate(geom, r, r, x4, launch)
    torch.cuda.synchronize()
    assert s64.device_status() == 0 and s32.device_status() == 0
    assert torch.equal(x1, x2)
    assert torch.equal(x3, x4)


@pytest.mark.parametrize("tensor_cores", [False, True])
def test_fused_defect_correction_equals_unfused(tcs, tensor_cores):
    """The fused period (defect sweep, first correction step read from r, accumulating last step)
    gives the unfused period's state bit for bit."""
    import torch

    from threadcoarsenedstencilgenerator_b200.mixed import DefectCorrectedSweeps

    cfg = (2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0)
    spec = G.spec_of(cfg)
    geom = spec.geometry(520, 300)
    rng = np.random.default_rng(23)
    mask = rng.standard_normal(spec.stencil_size) / spec.stencil_size
    a = rng.uniform(-1, 1, geom.shape)
    launch = tcs.Launch(block=(32, 1, 1), variant="pipe")
    out = []
    for fused in (True, False):
        dc = DefectCorrectedSweeps(spec, launch, mask=mask, tensor_cores=tensor_cores, fused=fused)
        x = torch.from_numpy(a).cuda()
        x, res = dc.run(geom, x, 45, 20)
        torch.cuda.synchronize()
        assert dc.fused == fused
        out.append((x.cpu(), res))
    assert torch.equal(out[0][0], out[1][0])
    assert out[0][1].fp64_sweeps == out[1][1].fp64_sweeps == 3
    for (m0, l0), (m1, l1) in zip(out[0][1].residual_history, out[1][1].residual_history):
        assert m0 == m1 and abs(l0 - l1) <= 1e-12 * l1
