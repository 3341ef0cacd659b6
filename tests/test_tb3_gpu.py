"""Temporal blocking in 3D and 2D (two sweeps per pass, tcs_sweeps_tb3) against the oracle, bit for
bit: several parameter sets and launch shapes, FP64 and FP32, odd sweep counts (the last sweep is
an ordinary one), partial last tiles and strips, a Read/Write padded row pitch, and the 2D
configuration-1 grid (Box Jacobi r1, 4096 x 4096) at full size."""

import numpy as np
import pytest

import gpu_util as G
import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    # (cfg, precision, sides, launch block or None)
    ((3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0), "f64", (70, 61, 40), None),
    ((3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0), "f32", (83, 45, 33), None),
    ((3, "Star", "Row", "Variable", 4, 2, 4, 1, "Read", 16), "f64", (150, 75, 37), None),
    ((3, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0), "f64", (77, 70, 29), None),
    ((3, "Box", "Column", "Variable", 1, 2, 1, 1, "Write", 8), "f64", (61, 40, 25), (16, 16)),
    ((3, "Star", "Column", "Variable", 3, 1, 1, 1, "Write", 8), "f64", (55, 50, 31), (32, 16)),
    ((3, "Box", "Row", "Variable", 2, 2, 2, 1, "None", 0), "f32", (90, 44, 21), (16, 8)),
    # 2D strips marching along y
    ((2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0), "f64", (1000, 700), None),
    ((2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0), "f64", (523, 611), (62, 1)),
    ((2, "Star", "Row", "Variable", 2, 2, 1, 1, "Read", 8), "f64", (700, 400), None),
    ((2, "Star", "Row", "Jacobi", 2, 1, 1, 1, "None", 0), "f32", (777, 300), None),
    ((2, "Box", "Row", "Variable", 3, 1, 1, 1, "Write", 8), "f64", (600, 300), (94, 1)),
    ((2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0), "f64", (900, 260), None),
]


@pytest.fixture(scope="module")
def tcs():
    import threadcoarsenedstencilgenerator_b200 as t

    return t


@pytest.mark.parametrize("n", [2, 5])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "%s_%s_%s_r%d_%s" % (c[0][1], c[0][2], c[0][3], c[0][4], c[1]))
def test_tb3_equals_ordinary_sweeps(tcs, case, n):
    import torch

    cfg, prec, sides, block = case
    spec = G.spec_of(cfg, prec)
    st = tcs.Stencil(spec)
    geom = spec.geometry(*sides)
    launch = None if block is None else tcs.Launch(block=tuple(block) + (1,) * (3 - len(block)))
    plan = st.plan_tb3(geom, launch)
    assert plan.variant == "tb3" and plan.grid_blocks[0] >= 1
    rng = np.random.default_rng(cfg[4] + n)
    dt = np.float64 if prec == "f64" else np.float32
    a = rng.uniform(-1, 1, geom.shape).astype(dt)
    mask = rng.standard_normal(spec.stencil_size) if cfg[3] == "Variable" else None
    if mask is not None:
        st.copy_mask(mask)
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    res = st.sweeps_tb3(geom, x, y, n, launch)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    want = O.sweeps(O.make_spec(*cfg), a, n, geom.right_offset, mask)
    assert np.array_equal(res.cpu().numpy(), want)


def test_tb3_work_split_does_not_change_results(tcs):
    """One CTA, a prime CTA count and the default split of the (tile, plane) work list give the
    same bits (pieces restart both pipelines at arbitrary planes)."""
    import torch

    cfg = (3, "Star", "Row", "Variable", 2, 2, 2, 1, "None", 0)
    spec = G.spec_of(cfg)
    st = tcs.Stencil(spec)
    geom = spec.geometry(100, 50, 30)
    rng = np.random.default_rng(3)
    a = rng.random(geom.shape)
    st.copy_mask(rng.standard_normal(spec.stencil_size))
    outs = []
    for segments in (0, 1, 7):
        x = torch.from_numpy(a).cuda()
        y = x.clone()
        res = st.sweeps_tb3(geom, x, y, 2, tcs.Launch(block=(32, 16, 1), segments=segments))
        torch.cuda.synchronize()
        outs.append(res.cpu())
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])


@pytest.mark.parametrize("segments", [1, 7])
def test_tb3_2d_work_split_does_not_change_results(tcs, segments):
    """2D strips: one CTA and a prime CTA count give the bits of the default split (pieces restart
    both pipelines at arbitrary rows)."""
    import torch

    cfg = (2, "Box", "Row", "Variable", 1, 1, 1, 1, "None", 0)
    spec = G.spec_of(cfg)
    st = tcs.Stencil(spec)
    geom = spec.geometry(530, 333)
    rng = np.random.default_rng(5)
    a = rng.random(geom.shape)
    st.copy_mask(rng.standard_normal(spec.stencil_size))
    outs = []
    for seg in (0, segments):
        x = torch.from_numpy(a).cuda()
        y = x.clone()
        res = st.sweeps_tb3(geom, x, y, 2, tcs.Launch(block=(64, 1, 1), segments=seg))
        torch.cuda.synchronize()
        outs.append(res.cpu())
    assert st.device_status() == 0
    assert torch.equal(outs[0], outs[1])


def test_tb3_2d_full_size_box_jacobi_r1_4096():
    """The configuration-1 grid at full size: 4096 x 4096 FP64, two sweeps in one pass, default
    launch, against the oracle."""
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs

    cfg = (2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0)
    spec = G.spec_of(cfg)
    st = tcs.Stencil(spec)
    geom = spec.geometry(4096, 4096)
    rng = np.random.default_rng(2024)
    a = rng.random(geom.shape)
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    res = st.sweeps_tb3(geom, x, y, 2)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    want = O.sweeps(O.make_spec(*cfg), a, 2, geom.right_offset, None)
    assert np.array_equal(res.cpu().numpy(), want)


def test_tb3_rejects_what_it_cannot_run(tcs):
    import torch

    st2 = tcs.Stencil(tcs.StencilSpec(dimension=2, neighbourhood="Star", orientation="Column", range=1))
    g2 = st2.spec.geometry(40, 40)
    x2 = torch.zeros(g2.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(tcs.UnsupportedLaunch):
        st2.sweeps_tb3(g2, x2, x2.clone(), 2)
    # FP32 with an odd range: no output tile of 16-byte multiples
    st = tcs.Stencil(tcs.StencilSpec(dimension=3, neighbourhood="Star", range=1, precision="f32"))
    g = st.spec.geometry(40, 40, 40)
    x = torch.zeros(g.shape, dtype=torch.float32, device="cuda")
    with pytest.raises(tcs.UnsupportedLaunch):
        st.sweeps_tb3(g, x, x.clone(), 2)
