"""Compensated FP32 accumulation (precision "f32c") against the float64 oracle.

Every output sums its terms in the reference's order with two-sum error terms for the additions
and fma(v, m, -v*m) for the products, so the result is the correctly summed value rounded once or
twice: |f32c - exact| <= 3 * 2^-24 * |exact| (two roundings of the final value, and for Jacobi the
FP32 weight fl(1/S)) + 4 * S * 2^-48 * sum |mask| |in| (the error terms are summed in FP32 too).  "exact" is the float64 oracle on the same
FP32 inputs and FP32-rounded mask.  Plain FP32 must do worse on the long stencil.
"""

import numpy as np
import pytest

import gpu_util as G
import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    ((2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0), (32, 4, 1), (301, 207, 1)),
    ((3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16), (32, 4, 1), (60, 44, 38)),
    ((2, "Box", "Column", "Jacobi", 3, 2, 2, 1, "None", 0), (16, 8, 1), (150, 99, 1)),
    ((3, "Box", "Row", "Variable", 2, 1, 2, 2, "Write", 8), (32, 2, 2), (41, 37, 29)),
]


@pytest.fixture(scope="module")
def tcs():
    import threadcoarsenedstencilgenerator_b200 as t

    return t


@pytest.mark.parametrize("variant", ["direct", "march"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "%dD_%s_%s_%s_r%d" % (c[0][0], c[0][1], c[0][2], c[0][3], c[0][4]))
def test_compensated_fp32_is_within_rounding_of_fp64(tcs, case, variant):
    import torch

    cfg, block, sides = case
    rng = np.random.default_rng(cfg[4])
    out = {}
    for prec in ("f32c", "f32"):
        spec = G.spec_of(cfg, prec)
        st = tcs.Stencil(spec)
        geom = spec.geometry(*sides[:cfg[0]])
        if prec == "f32c":
            a = rng.uniform(-1, 1, geom.shape).astype(np.float32)
            mask = rng.standard_normal(spec.stencil_size) / spec.stencil_size if cfg[3] == "Variable" else None
        if mask is not None:
            st.copy_mask(mask)
        x = torch.from_numpy(a).cuda()
        y = x.clone()
        try:
            st.update_grid(geom, x, y, tcs.Launch(block=block, variant=variant))
        except tcs.UnsupportedLaunch:
            pytest.skip("%s does not run this shape" % variant)
        torch.cuda.synchronize()
        assert st.device_status() == 0
        out[prec] = y.cpu().numpy().astype(np.float64)
    m32 = None if mask is None else mask.astype(np.float32).astype(np.float64)
    exact = O.sweep(O.make_spec(*cfg), a.astype(np.float64), geom.right_offset, m32)
    sl = geom.interior_slices(cfg[4])
    err_c = np.abs(out["f32c"][sl] - exact[sl])
    err_p = np.abs(out["f32"][sl] - exact[sl])
    # second-order part: the error terms are themselves summed in FP32 (S terms of size <= eps * term)
    absm = None if m32 is None else np.abs(m32)
    mag = O.sweep(O.make_spec(*cfg), np.abs(a.astype(np.float64)), geom.right_offset, absm)[sl]
    S = G.spec_of(cfg).stencil_size
    bound = 3 * 2.0 ** -24 * np.abs(exact[sl]) + 4 * S * 2.0 ** -48 * mag
    assert np.all(err_c <= bound), float((err_c / bound).max())
    if cfg[3] == "Variable" and cfg[4] >= 4:
        assert err_c.max() < err_p.max()
    # padding and border untouched
    outside = np.ones(geom.shape, dtype=bool)
    outside[sl] = False
    assert np.array_equal(out["f32c"][outside], a.astype(np.float64)[outside])


def test_compensated_fp32_rejects_the_pipe_kernel(tcs):
    import torch

    spec = tcs.StencilSpec(dimension=3, neighbourhood="Star", coefficients="Variable", range=2, cx=2, cy=2,
                           precision="f32c")
    st = tcs.Stencil(spec)
    geom = spec.geometry(40, 40, 40)
    x = torch.zeros(geom.shape, dtype=torch.float32, device="cuda")
    with pytest.raises(tcs.UnsupportedLaunch):
        st.update_grid(geom, x, x.clone(), tcs.Launch(block=(16, 4, 1), variant="pipe"))
    st.update_grid(geom, x, x.clone(), tcs.Launch(block=(16, 4, 1)))  # auto: march or direct


PIPE_COMP_CASES = [
    ((2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0), (32, 1, 1), (301, 207, 1)),
    ((2, "Box", "Row", "Jacobi", 3, 8, 1, 1, "Read", 16), (32, 1, 1), (400, 90, 1)),
    ((3, "Box", "Row", "Variable", 2, 2, 2, 1, "Read", 16), (32, 4, 1), (90, 44, 30)),
]


@pytest.mark.parametrize("case", PIPE_COMP_CASES, ids=lambda c: "%dD_%s_%s_r%d_c%d" % (c[0][0], c[0][1], c[0][3], c[0][4], c[0][5]))
def test_pipe_compensated_rows_within_bound(tcs, case):
    """The pipelined kernel's compensated FP32 form (packed Box path, row partials combined by
    two-sum): |f32c - exact| <= 3u|exact| + (2R + 2) u sum|mask||in| per point (u = 2^-24), and
    better than plain FP32 on Variable stencils."""
    import torch

    cfg, block, sides = case
    rng = np.random.default_rng(40 + cfg[4])
    out = {}
    S = G.spec_of(cfg).stencil_size
    for prec in ("f32c", "f32"):
        spec = G.spec_of(cfg, prec)
        st = tcs.Stencil(spec)
        geom = spec.geometry(*sides[:cfg[0]])
        if prec == "f32c":
            a = rng.uniform(-1, 1, geom.shape).astype(np.float32)
            mask = rng.standard_normal(S) / S if cfg[3] == "Variable" else None
        if mask is not None:
            st.copy_mask(mask)
        launch = tcs.Launch(block=block, variant="pipe")
        assert st.plan(geom, launch).variant == "pipe"
        x = torch.from_numpy(a).cuda()
        y = x.clone()
        st.sweeps(geom, x, y, 1, launch)
        torch.cuda.synchronize()
        assert st.device_status() == 0
        out[prec] = y.cpu().numpy().astype(np.float64)
    m32 = None if mask is None else mask.astype(np.float32).astype(np.float64)
    exact = O.sweep(O.make_spec(*cfg), a.astype(np.float64), geom.right_offset, m32)
    absm = None if m32 is None else np.abs(m32)
    mag = O.sweep(O.make_spec(*cfg), np.abs(a.astype(np.float64)), geom.right_offset, absm)
    if cfg[3] == "Jacobi":  # FP32 sweeps scale by fl32(1/S)
        f = np.float64(np.float32(1.0 / S)) * S
        exact, mag = exact * f, mag * f
    sl = geom.interior_slices(cfg[4])
    u = 2.0 ** -24
    bound = 3 * u * np.abs(exact[sl]) + (2 * cfg[4] + 2) * u * mag[sl]
    err = np.abs(out["f32c"][sl] - exact[sl])
    assert np.all(err <= bound), float((err / bound).max())
    if cfg[3] == "Variable":
        assert err.max() < np.abs(out["f32"][sl] - exact[sl]).max()
    outside = np.ones(geom.shape, dtype=bool)
    outside[sl] = False
    assert np.array_equal(out["f32c"][outside], a.astype(np.float64)[outside])
