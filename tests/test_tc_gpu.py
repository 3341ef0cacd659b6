"""Tensor-core sweep of 2D Box stencils (tcs_tc_update_grid) against the float64 oracle.

The sweep splits inputs and mask into BF16 high and low parts and accumulates hi*hi + hi*lo +
lo*hi in FP32.  Per product the dropped lo*lo term and the BF16 rounding of the low parts are
below 2^-16 of |mask * in|, and FP32 accumulation over at most 289 terms adds well under 2^-15, so
the test bound is |tc - oracle| <= 4e-5 * sum |mask| |in| at every interior point.  Points outside
the interior must keep their values.
"""

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _spec(tcs, R, coeff="Variable"):
    return tcs.StencilSpec(dimension=2, neighbourhood="Box", coefficients=coeff, range=R, precision="f32")


@pytest.fixture(scope="module")
def tcs():
    import threadcoarsenedstencilgenerator_b200 as t

    return t


@pytest.mark.parametrize("R, shape", [(1, (300, 200)), (3, (517, 1000)), (6, (1100, 389)), (8, (333, 777))])
def test_tc_sweep_within_bound_of_fp64_oracle(tcs, R, shape):
    import torch

    spec = _spec(tcs, R)
    st = tcs.Stencil(spec)
    geom = spec.geometry(*shape)
    rng = np.random.default_rng(R)
    S = spec.stencil_size
    mask = rng.standard_normal(S) / S
    st.copy_mask(mask)
    a = rng.uniform(-1, 1, geom.shape).astype(np.float32)
    src = rng.uniform(-1e-3, 1e-3, geom.shape).astype(np.float32)
    x = torch.from_numpy(a).cuda()
    s = torch.from_numpy(src).cuda()
    y = torch.full(geom.shape, 7.0, dtype=torch.float32, device="cuda")
    for with_src in (False, True):
        st.tc_update_grid(geom, x, y, source=s if with_src else None)
        torch.cuda.synchronize()
        got = y.cpu().numpy().astype(np.float64)
        ospec = O.make_spec(2, "Box", "Row", "Variable", R, 1, 1)
        want = O.sweep(ospec, a.astype(np.float64), geom.right_offset, mask)
        bound = O.sweep(ospec, np.abs(a.astype(np.float64)), geom.right_offset, np.abs(mask))
        sl = geom.interior_slices(R)
        if with_src:
            want[sl] += src.astype(np.float64)[sl]
        err = np.abs(got[sl] - want[sl])
        assert np.all(err <= 4e-5 * bound[sl] + 1e-7), float((err / (bound[sl] + 1e-30)).max())
        outside = np.ones(geom.shape, dtype=bool)
        outside[sl] = False
        assert np.all(got[outside] == 7.0)
    assert st.device_status() == 0


def test_tc_jacobi_and_mask_update(tcs):
    """Jacobi weights 1/S; a new mask takes effect on the next sweep."""
    import torch

    R = 2
    spec = _spec(tcs, R, "Jacobi")
    st = tcs.Stencil(spec)
    geom = spec.geometry(260, 140)
    a = np.random.default_rng(1).uniform(0, 1, geom.shape).astype(np.float32)
    x = torch.from_numpy(a).cuda()
    y = torch.zeros_like(x)
    st.tc_update_grid(geom, x, y)
    torch.cuda.synchronize()
    ospec = O.make_spec(2, "Box", "Row", "Jacobi", R, 1, 1)
    want = O.sweep(ospec, a.astype(np.float64), geom.right_offset)
    sl = geom.interior_slices(R)
    assert np.max(np.abs(y.cpu().numpy()[sl] - want[sl])) <= 4e-5
    vspec = _spec(tcs, R)
    sv = tcs.Stencil(vspec)
    for seed in (2, 3):
        mask = np.random.default_rng(seed).standard_normal(vspec.stencil_size)
        sv.copy_mask(mask)
        sv.tc_update_grid(geom, x, y)
        torch.cuda.synchronize()
        want = O.sweep(O.make_spec(2, "Box", "Row", "Variable", R, 1, 1), a.astype(np.float64), geom.right_offset, mask)
        bound = O.sweep(O.make_spec(2, "Box", "Row", "Variable", R, 1, 1), np.abs(a.astype(np.float64)),
                        geom.right_offset, np.abs(mask))
        assert np.all(np.abs(y.cpu().numpy()[sl] - want[sl]) <= 4e-5 * bound[sl] + 1e-7)


def test_tc_rejects_unsupported_parameter_sets(tcs):
    for kw in (dict(dimension=3, neighbourhood="Box", range=2, precision="f32"),
               dict(dimension=2, neighbourhood="Star", range=2, precision="f32"),
               dict(dimension=2, neighbourhood="Box", range=2, precision="f64"),
               dict(dimension=2, neighbourhood="Box", range=9, precision="f32")):
        st = tcs.Stencil(tcs.StencilSpec(**kw))
        g = st.spec.geometry(64, 64, 64) if kw["dimension"] == 3 else st.spec.geometry(64, 64)
        import torch

        dt = torch.float32 if kw["precision"] == "f32" else torch.float64
        x = torch.zeros(g.shape, dtype=dt, device="cuda")
        with pytest.raises(tcs.UnsupportedLaunch):
            st.tc_update_grid(g, x, x.clone())


def test_tc_defect_corrected_iteration_tracks_fp64(tcs):
    """200 sweeps of 2D Box Variable r6 as tensor-core FP32 sweeps with FP64 defect correction every
    20: max and RMS relative error against the FP64 sweeps <= 1e-6."""
    import torch

    from threadcoarsenedstencilgenerator_b200.mixed import DefectCorrectedSweeps

    spec = tcs.StencilSpec(dimension=2, neighbourhood="Box", coefficients="Variable", range=6)
    geom = spec.geometry(700, 420)
    rng = np.random.default_rng(4)
    mask = rng.standard_normal(spec.stencil_size) / spec.stencil_size
    a = rng.uniform(-1, 1, geom.shape)
    ref = tcs.Stencil(spec)
    ref.copy_mask(mask)
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    want = ref.sweeps(geom, x, y, 200, tcs.Launch(block=(32, 4, 1), variant="direct"))
    dc = DefectCorrectedSweeps(spec, tcs.Launch(block=(32, 4, 1), variant="direct"), mask=mask, tensor_cores=True)
    xm = torch.from_numpy(a).cuda()
    xm, res = dc.run(geom, xm, 200, period=20)
    st = dc.s64.compare(geom, xm, want, "f64")
    assert st["max_rel"] <= 1e-6 and st["rms_rel"] <= 1e-6, st
