"""Ragged grids (interior not a multiple of the coarsening): every interior point is swept.

The expected values are the oracle's sweeps of the same buffers with coarsening 1 -- the
per-point term order does not depend on the coarsening, so a ragged sweep must equal them bit for
bit (the kernels sweep the whole coarsening tiles, a coarsening-1 direct instance the fringe).
Padding and borders keep their values.
"""

import numpy as np
import pytest

import gpu_util as G
import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    ((3, "Star", "Row", "Variable", 4, 2, 4, 3, "Read", 16), (16, 4, 1), (61, 47, 39)),
    ((2, "Box", "Row", "Variable", 3, 4, 3, 1, "None", 0), (16, 4, 1), (103, 77, 1)),
    ((3, "Box", "Column", "Jacobi", 1, 2, 2, 2, "Write", 8), (16, 4, 1), (33, 29, 27)),
    ((2, "Star", "Column", "Variable", 2, 3, 2, 1, "Read", 8), (32, 4, 1), (92, 59, 1)),
]


@pytest.fixture(scope="module")
def tcs():
    import threadcoarsenedstencilgenerator_b200 as t

    return t


@pytest.mark.parametrize("variant", ["direct", "march", "pipe", "auto"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "%dD_%s_%s_r%d" % (c[0][0], c[0][1], c[0][3], c[0][4]))
def test_ragged_sweep_equals_coarsening_one_oracle(tcs, case, variant):
    import torch

    cfg, block, sides = case
    spec = G.spec_of(cfg)
    st = tcs.Stencil(spec)
    geom = spec.geometry(*sides[:cfg[0]], ragged=True)
    assert geom.grid[:cfg[0]] != spec.geometry(*sides[:cfg[0]]).grid[:cfg[0]]  # really ragged
    rng = np.random.default_rng(cfg[4] + cfg[5])
    a = rng.uniform(-1, 1, geom.shape)
    mask = rng.standard_normal(spec.stencil_size) if cfg[3] == "Variable" else None
    if mask is not None:
        st.copy_mask(mask)
    b3 = block if cfg[0] == 3 else (block[0], block[1], 1)
    if variant == "pipe":  # pipe blocks: (bx, by, 1) in 3D, (bx, 1, 1) in 2D
        b3 = (block[0], block[1] if cfg[0] == 3 else 1, 1)
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    try:
        res = st.sweeps(geom, x, y, 2, tcs.Launch(block=b3, variant=variant))
    except tcs.UnsupportedLaunch:
        pytest.skip("%s does not run this shape" % variant)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    want = O.sweeps(O.make_spec(d, sh, o, c, r, 1, 1, 1, al, cl), a, 2, geom.right_offset, mask)
    assert np.array_equal(res.cpu().numpy(), want)


def test_ragged_batch(tcs):
    """Batched sweeps of ragged grids: every grid equals its coarsening-1 oracle sweeps."""
    import torch

    from threadcoarsenedstencilgenerator_b200.batch import BatchedSweeps

    cfg = (3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0)
    spec = G.spec_of(cfg)
    st = tcs.Stencil(spec)
    sides = [(41, 23, 19), (18, 30, 26), (27, 19, 35)]
    geoms = [spec.geometry(*s, ragged=True) for s in sides]
    rng = np.random.default_rng(8)
    arrs = [rng.random(g.shape) for g in geoms]
    xs = [torch.from_numpy(v).cuda() for v in arrs]
    ys = [v.clone() for v in xs]
    bt = BatchedSweeps(st, geoms, xs, ys, tcs.Launch(block=(16, 4, 1), variant="pipe"))
    res = bt.sweeps(3)
    torch.cuda.synchronize()
    ospec = O.make_spec(3, "Star", "Row", "Jacobi", 2, 1, 1, 1)
    for g, v, r in zip(geoms, arrs, res):
        assert np.array_equal(r.cpu().numpy(), O.sweeps(ospec, v, 3, g.right_offset))
    bt.close()
