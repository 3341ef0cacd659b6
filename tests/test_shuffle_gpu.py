"""Star middle rows through warp shuffles (TCS_LAUNCH_SHUFFLE) against the oracle, bit for bit.

The shuffles only move values between lanes, so the results must equal the oracle at 0 ulp:
several ranges (halos of one, two and up to eight neighbour lanes), coarsenings, 2D and 3D,
FP64 and FP32, Read/Write padding, partial last tiles, and the benchmarked 512^3 instantiation."""

import numpy as np
import pytest

import gpu_util as G
import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    # (cfg, block, sides)
    ((3, "Star", "Row", "Variable", 4, 2, 4, 1, "Read", 16), (64, 4, 1), (300, 75, 37)),
    ((3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16), (64, 8, 1), (150, 70, 30)),
    ((3, "Star", "Row", "Jacobi", 2, 2, 2, 1, "None", 0), (32, 8, 1), (101, 50, 31)),
    ((3, "Star", "Row", "Variable", 3, 2, 1, 1, "Write", 8), (32, 4, 1), (90, 33, 21)),
    ((3, "Star", "Row", "Jacobi", 1, 1, 4, 1, "None", 0), (32, 4, 1), (77, 60, 19)),
    ((2, "Star", "Row", "Variable", 3, 2, 1, 1, "Read", 16), (32, 1, 1), (333, 120, 1)),
    ((2, "Star", "Row", "Jacobi", 8, 1, 1, 1, "None", 0), (64, 1, 1), (300, 80, 1)),
]


@pytest.fixture(scope="module")
def tcs():
    import threadcoarsenedstencilgenerator_b200 as t

    return t


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "%dD_%s_r%d_c%dx%d_b%dx%d" % (c[0][0], c[0][3], c[0][4], c[0][5],
                                                                                 c[0][6], c[1][0], c[1][1]))
def test_shuffled_rows_match_oracle(tcs, case, precision):
    import torch

    cfg, block, sides = case
    spec = G.spec_of(cfg, precision)
    st = tcs.Stencil(spec)
    geom = spec.geometry(*sides[:cfg[0]])
    launch = tcs.Launch(block=block, variant="pipe", shuffle=True)
    assert st.plan(geom, launch).variant == "pipe"
    rng = np.random.default_rng(cfg[4] * 7 + len(precision))
    dt = np.float64 if precision == "f64" else np.float32
    a = rng.uniform(-1, 1, geom.shape).astype(dt)
    mask = rng.standard_normal(spec.stencil_size) if cfg[3] == "Variable" else None
    if mask is not None:
        st.copy_mask(mask)
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    res = st.sweeps(geom, x, y, 3, launch)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    assert np.array_equal(res.cpu().numpy(), O.sweeps(O.make_spec(*cfg), a, 3, geom.right_offset, mask))


def test_shuffled_rows_full_workload(tcs):
    """The 512^3 Star Variable r4 workload with shuffled rows, two sweeps: the register pipeline's
    best shape (2x4 tiles, 64x4 blocks, 3 planes per chunk; shuffles are a register-pipeline
    option, the tuned launch runs the ring form)."""
    import torch

    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    w = WORKLOADS["3d_star_var_r4_512"]
    spec = w.spec.replace(cx=2, cy=4, cz=1)
    launch = tcs.Launch(block=(64, 4, 1), variant="pipe", chunk=3, shuffle=True)
    geom = spec.geometry(*w.grid)
    st = tcs.Stencil(spec)
    mask = w.make_mask()
    st.copy_mask(mask)
    a = w.make_input(geom)
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    res = st.sweeps(geom, x, y, 2, launch)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    want = O.sweeps(O.make_spec(spec.dimension, spec.neighbourhood, spec.orientation, spec.coefficients, spec.range,
                                spec.cx, spec.cy, spec.cz, spec.alignment, spec.cl_size), a, 2, geom.right_offset,
                    mask, cpu_threads=0)
    assert np.array_equal(res.cpu().numpy(), want)


def test_shuffle_request_rejected_where_it_cannot_apply(tcs):
    import torch

    spec = tcs.StencilSpec(dimension=3, neighbourhood="Box", range=1, cx=2)
    st = tcs.Stencil(spec)
    g = spec.geometry(70, 40, 20)
    x = torch.zeros(g.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(tcs.UnsupportedLaunch):
        st.update_grid(g, x, x.clone(), tcs.Launch(block=(32, 4, 1), variant="pipe", shuffle=True))
