"""The ring form of the pipelined sweep (own centre values and finished crosses in tensor memory,
TCS_LAUNCH_TMEM) against the oracle on the GPU, bit for bit.

Cases: 3D Star stencils in Row order, FP64 and FP32, ranges 1-5, several coarsenings and blocks,
mid-size grids with ragged last tiles and with more tiles than CTAs (so CTAs sweep pieces that
restart the rings from stale contents), several sweeps; and the 3D Star Variable r4 512^3
workload's own grid and data for two sweeps.
"""

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tcs():
    import torch

    import threadcoarsenedstencilgenerator_b200 as t

    assert torch.cuda.is_available()
    return t


def _spec(tcs, cfg, precision):
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    return tcs.StencilSpec(dimension=d, neighbourhood=sh, orientation=o, coefficients=c, range=r, cx=cx, cy=cy,
                           cz=cz, alignment=al, cl_size=cl, precision=precision)


def _run(tcs, spec, geom, a, mask, n, launch):
    import torch

    st = tcs.Stencil(spec)
    if mask is not None:
        st.copy_mask(mask)
    plan = st.plan(geom, launch)
    assert plan.variant == "pipe"
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    res = st.sweeps(geom, x, y, n, launch)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    out = res.cpu().numpy()
    st.close()
    return out, plan


CASES = [
    # cfg, block, chunk
    ((3, "Star", "Row", "Variable", 4, 2, 4, 1, "Read", 16), (64, 4), 1),
    ((3, "Star", "Row", "Variable", 4, 2, 4, 1, "Read", 16), (64, 2), 2),
    ((3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16), (64, 8), 1),
    ((3, "Star", "Row", "Jacobi", 1, 1, 4, 1, "None", 0), (128, 2), 3),
    ((3, "Star", "Row", "Variable", 2, 2, 4, 1, "Write", 8), (32, 4), 1),
    ((3, "Star", "Row", "Jacobi", 3, 2, 4, 1, "None", 0), (32, 8), 2),
    ((3, "Star", "Row", "Variable", 5, 2, 2, 1, "Read", 16), (64, 4), 1),
]


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "r%d_%dx%d_b%dx%d_ch%d" % (c[0][4], c[0][5], c[0][6], *c[1], c[2]))
def test_ring_form_matches_oracle(tcs, case, precision):
    cfg, (bx, by), ch = case
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec = _spec(tcs, cfg, precision)
    tx, ty = bx * cx, by * cy
    geom = spec.geometry(2 * r + 3 * tx + 5 * cx + 3, 2 * r + 3 * ty + 3 * cy + 1, 2 * r + 41)
    rng = np.random.default_rng(21)
    dt = np.float64 if precision == "f64" else np.float32
    a = rng.random(geom.shape).astype(dt)
    mask = rng.standard_normal(spec.stencil_size) if c == "Variable" else None
    launch = tcs.Launch(block=(bx, by, 1), variant="pipe", chunk=ch, tmem=True)
    got, plan = _run(tcs, spec, geom, a, mask, 4, launch)
    want = O.sweeps(O.make_spec(*cfg), a, 4, geom.right_offset, mask)
    assert np.array_equal(got, want), "max |diff| %g" % float(np.abs(got.astype(np.float64) - want).max())


def test_ring_form_workload_grid_matches_oracle(tcs):
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    w = WORKLOADS["3d_star_var_r4_512"]
    spec = w.spec.replace(cx=2, cy=4, cz=1)
    geom = spec.geometry(*w.grid)
    a = w.make_input(geom)
    mask = w.make_mask()
    launch = tcs.Launch(block=(64, 4, 1), variant="pipe", chunk=1, tmem=True)
    got, plan = _run(tcs, spec, geom, a, mask, 2, launch)
    want = O.sweeps(O.make_spec(3, "Star", "Row", "Variable", 4, 2, 4, 1, "Read", 16), a, 2, geom.right_offset,
                    mask, cpu_threads=0)
    assert np.array_equal(got, want)


def test_ring_form_rejected_where_it_does_not_apply(tcs):
    spec = _spec(tcs, (3, "Box", "Row", "Variable", 2, 2, 2, 1, "Read", 16), "f64")
    st = tcs.Stencil(spec)
    with pytest.raises(tcs.UnsupportedLaunch):
        st.plan(spec.geometry(96, 64, 40), tcs.Launch(block=(32, 4, 1), variant="pipe", chunk=1, tmem=True))
    st.close()


LOCKSTEP_CASES = [
    # cfg, block, chunk, ring form
    ((3, "Star", "Row", "Variable", 4, 2, 4, 1, "Read", 16), (64, 7), 2, True),
    ((3, "Star", "Row", "Variable", 4, 2, 4, 1, "Read", 16), (32, 7), 3, False),
    ((3, "Box", "Row", "Variable", 2, 2, 2, 1, "Write", 8), (32, 4), 2, False),
    ((3, "Star", "Row", "Jacobi", 3, 2, 2, 1, "None", 0), (64, 6), 3, True),
]


@pytest.mark.parametrize("case", LOCKSTEP_CASES,
                         ids=lambda c: "%s_r%d_b%dx%d_ch%d_%s" % (c[0][1], c[0][4], *c[1], c[2], "ring" if c[3] else "reg"))
def test_lockstep_matches_oracle(tcs, case):
    """Lockstep CTAs (whole tile columns or equal parts of one) give the same bits: grids whose tile
    count does not divide the resident CTAs, whose march length does not divide into the parts
    (pieces straddle tile columns), with ragged last tiles."""
    cfg, (bx, by), ch, ring = case
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec = _spec(tcs, cfg, "f64")
    tx, ty = bx * cx, by * cy
    geom = spec.geometry(2 * r + 2 * tx + 3 * cx + 1, 2 * r + 3 * ty + cy + 1, 2 * r + 53)
    rng = np.random.default_rng(23)
    a = rng.random(geom.shape)
    mask = rng.standard_normal(spec.stencil_size) if c == "Variable" else None
    launch = tcs.Launch(block=(bx, by, 1), variant="pipe", chunk=ch, tmem=ring, lockstep=True)
    got, plan = _run(tcs, spec, geom, a, mask, 3, launch)
    tiles = -(-geom.elements[0] // tx) * -(-geom.elements[1] // ty)
    assert plan.grid_blocks[0] <= tiles * max(1, plan.num_sms * plan.ctas_per_sm // tiles)
    want = O.sweeps(O.make_spec(*cfg), a, 3, geom.right_offset, mask)
    assert np.array_equal(got, want), "max |diff| %g" % float(np.abs(got - want).max())
