"""Temporal blocking (two sweeps per pass, tcs_sweeps_tb2) against the oracle, bit for bit."""

import numpy as np
import pytest

import gpu_util as G
import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    ((2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0), "f64", (300, 200), False),
    ((2, "Box", "Row", "Variable", 3, 2, 2, 1, "Read", 16), "f64", (517, 300), False),
    ((2, "Star", "Column", "Variable", 2, 1, 2, 1, "Write", 8), "f64", (261, 180), False),
    ((2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0), "f32", (400, 333), False),
    ((2, "Box", "Row", "Variable", 3, 4, 3, 1, "None", 0), "f64", (103, 77), True),
    ((2, "Star", "Row", "Jacobi", 8, 1, 1, 1, "None", 0), "f64", (291, 170), True),
    ((2, "Box", "Column", "Jacobi", 1, 2, 2, 1, "None", 0), "f32", (7, 5), False),
]


@pytest.fixture(scope="module")
def tcs():
    import threadcoarsenedstencilgenerator_b200 as t

    return t


@pytest.mark.parametrize("n", [1, 2, 5])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "%s_%s_r%d_%s%s" % (c[0][1], c[0][3], c[0][4], c[1],
                                                                          "_ragged" if c[3] else ""))
def test_tb2_equals_ordinary_sweeps(tcs, case, n):
    import torch

    cfg, prec, sides, ragged = case
    spec = G.spec_of(cfg, prec)
    st = tcs.Stencil(spec)
    geom = spec.geometry(*sides, ragged=ragged)
    rng = np.random.default_rng(cfg[4] + n)
    dt = np.float64 if prec == "f64" else np.float32
    a = rng.uniform(-1, 1, geom.shape).astype(dt)
    mask = rng.standard_normal(spec.stencil_size) if cfg[3] == "Variable" else None
    if mask is not None:
        st.copy_mask(mask)
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    res = st.sweeps_tb2(geom, x, y, n)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    want = O.sweeps(O.make_spec(d, sh, o, c, r, 1, 1, 1, al, cl), a, n, geom.right_offset, mask)
    assert np.array_equal(res.cpu().numpy(), want)


def test_tb2_rejects_3d(tcs):
    import torch

    spec = tcs.StencilSpec(dimension=3, neighbourhood="Star", range=1)
    st = tcs.Stencil(spec)
    g = spec.geometry(20, 20, 20)
    x = torch.zeros(g.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(tcs.UnsupportedLaunch):
        st.sweeps_tb2(g, x, x.clone(), 2)
