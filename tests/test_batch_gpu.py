"""Batched sweeps (one persistent launch over many grids) against the oracle and against
single-grid launches.

Small batches: every grid of the batch, after n ping-pong sweeps, equals n oracle sweeps of that
grid bit for bit (0 ulp, FP64 and FP32).  Full size (64 grids, sides log-uniform in [64, 256],
50 sweeps in a CUDA graph): the batched graph equals the same sweeps as one launch per grid, bit
for bit -- a size-independent property, since the single-grid path is itself pinned to the oracle.
"""

import numpy as np
import pytest

import gpu_util as G
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tcs():
    import threadcoarsenedstencilgenerator_b200 as t

    return t


def _upload(arrs):
    import torch

    xs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrs]
    ys = [x.clone() for x in xs]
    return xs, ys


BATCH_CASES = [
    # (cfg, block, sides)
    ((3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0), (16, 4, 1),
     [(40, 22, 18), (18, 30, 26), (26, 18, 34), (64, 40, 12), (22, 22, 22), (12, 14, 16)]),
    ((3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16), (16, 2, 1),
     [(45, 33, 20), (21, 17, 29), (60, 24, 18)]),
    ((3, "Box", "Row", "Variable", 1, 1, 2, 1, "None", 0), (32, 2, 1),
     [(35, 19, 9), (67, 11, 13), (20, 20, 20), (9, 9, 9)]),
    ((2, "Box", "Row", "Variable", 3, 4, 1, 1, "None", 0), (16, 1, 1),
     [(70, 41, 1), (133, 20, 1), (19, 97, 1), (40, 7, 1), (256, 64, 1)]),
]


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("case", BATCH_CASES, ids=lambda c: "%dD_%s_%s_r%d" % (c[0][0], c[0][1], c[0][3], c[0][4]))
def test_batch_matches_oracle_per_grid(tcs, case, precision):
    import torch

    from threadcoarsenedstencilgenerator_b200.batch import BatchedSweeps

    cfg, block, sides = case
    spec = G.spec_of(cfg, precision)
    st = tcs.Stencil(spec)
    dt = np.float64 if precision == "f64" else np.float32
    rng = np.random.default_rng(11)
    geoms = [spec.geometry(*s) for s in sides]
    arrs = [rng.random(g.shape).astype(dt) for g in geoms]
    mask = rng.standard_normal(spec.stencil_size) if cfg[3] == "Variable" else None
    if mask is not None:
        st.copy_mask(mask)
    xs, ys = _upload(arrs)
    bt = BatchedSweeps(st, geoms, xs, ys, tcs.Launch(block=block, variant="pipe"))
    n = 3
    res = bt.sweeps(n)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    ospec = O.make_spec(*cfg)
    for g, a, r in zip(geoms, arrs, res):
        want = O.sweeps(ospec, a, n, g.right_offset, mask)
        assert np.array_equal(r.cpu().numpy(), want), g
    bt.close()


def test_batch_mixes_tma_and_cp_async_grids(tcs):
    """FP32 rows of 4k+2 points cannot use TMA; such grids stream through cp.async in the same
    launch as TMA grids."""
    import torch

    from threadcoarsenedstencilgenerator_b200.batch import BatchedSweeps

    cfg = (3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0)
    spec = G.spec_of(cfg, "f32")
    st = tcs.Stencil(spec)
    sides = [(34, 20, 18), (32, 20, 18), (66, 26, 14), (64, 30, 22)]
    geoms = [spec.geometry(*s) for s in sides]
    rng = np.random.default_rng(5)
    arrs = [rng.random(g.shape).astype(np.float32) for g in geoms]
    xs, ys = _upload(arrs)
    bt = BatchedSweeps(st, geoms, xs, ys, tcs.Launch(block=(16, 4, 1), variant="pipe"))
    assert bt.plan().loader == "mixed"
    res = bt.sweeps(4)
    torch.cuda.synchronize()
    ospec = O.make_spec(*cfg)
    for g, a, r in zip(geoms, arrs, res):
        assert np.array_equal(r.cpu().numpy(), O.sweeps(ospec, a, 4, g.right_offset))
    bt.close()


def test_batch_cta_count_does_not_change_results(tcs):
    """Any split of the work list over CTAs (1 CTA, a prime count, the default) gives the same bits."""
    import torch

    from threadcoarsenedstencilgenerator_b200.batch import BatchedSweeps

    cfg = (3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0)
    spec = G.spec_of(cfg, "f64")
    st = tcs.Stencil(spec)
    sides = [(40, 22, 18), (18, 30, 26), (26, 18, 34)]
    geoms = [spec.geometry(*s) for s in sides]
    rng = np.random.default_rng(9)
    arrs = [rng.random(g.shape) for g in geoms]
    outs = []
    for segments in (0, 1, 7, 1000):
        xs, ys = _upload(arrs)
        bt = BatchedSweeps(st, geoms, xs, ys, tcs.Launch(block=(16, 4, 1), variant="pipe", segments=segments))
        res = bt.sweeps(2)
        torch.cuda.synchronize()
        outs.append([r.cpu().numpy() for r in res])
        bt.close()
    for o in outs[1:]:
        for u, v in zip(outs[0], o):
            assert np.array_equal(u, v)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_full_batch_graph_equals_separate_launches(tcs, precision):
    """64 uneven 3D Star Jacobi r2 grids, 50 sweeps: batched CUDA graph == one launch per grid."""
    import torch

    from threadcoarsenedstencilgenerator_b200.batch import BatchedSweeps
    from threadcoarsenedstencilgenerator_b200.workloads import BATCH_WORKLOADS

    w = BATCH_WORKLOADS["batch_3d_star_jacobi_r2_64"]
    spec = w.spec.replace(precision=precision)
    st = tcs.Stencil(spec)
    geoms = w.geometries(spec)
    dt = np.float64 if precision == "f64" else np.float32
    arrs = w.make_inputs(geoms, dt)
    launch = w.tuned_launch(precision)
    xs, ys = _upload(arrs)
    bt = BatchedSweeps(st, geoms, xs, ys, launch)
    bt.capture(w.sweeps)
    res = bt.replay()
    torch.cuda.synchronize()
    batched = [r.cpu() for r in res]
    bt.close()
    del xs, ys, res
    xs, ys = _upload(arrs)
    bt = BatchedSweeps(st, geoms, xs, ys, launch)
    bt.capture(w.sweeps, separate=True)
    res = bt.replay()
    torch.cuda.synchronize()
    assert st.device_status() == 0
    for u, v in zip(batched, res):
        assert torch.equal(u, v.cpu())
    bt.close()
    # one grid of the workload, one sweep, against the oracle
    xs, ys = _upload(arrs[:1])
    bt = BatchedSweeps(st, geoms[:1], xs, ys, launch)
    r1 = bt.sweeps(1)
    torch.cuda.synchronize()
    want = O.sweep(O.make_spec(3, "Star", "Row", "Jacobi", 2, 2, 2, 2), arrs[0], geoms[0].right_offset)
    assert np.array_equal(r1[0].cpu().numpy(), want)
    bt.close()


def test_batch_rejects_bad_arguments(tcs):
    import torch

    from threadcoarsenedstencilgenerator_b200.batch import BatchedSweeps

    spec = G.spec_of((3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0), "f64")
    st = tcs.Stencil(spec)
    g = spec.geometry(20, 20, 20)
    x = torch.zeros(g.shape, dtype=torch.float64, device="cuda")
    with pytest.raises(tcs.CudaErrorInvalidValue):
        BatchedSweeps(st, [g], [x], [x])
    with pytest.raises(tcs.UnsupportedLaunch):
        BatchedSweeps(st, [g], [x], [x.clone()], tcs.Launch(block=(16, 4, 1), variant="direct"))
    with pytest.raises(ValueError):
        BatchedSweeps(st, [], [], [])


@pytest.mark.parametrize("cx, sides, offset, loader", [
    (2, (32, 20, 18), 0, "tma"),             # 128-byte rows: TMA
    (2, (34, 20, 18), 0, "cp.async pairs"),  # 136-byte rows: two floats per copy
    (2, (34, 20, 18), 1, "cp.async pairs"),  # same pitch, base 4 bytes off: single floats
    (1, (33, 20, 18), 0, "cp.async"),        # odd pitch: single floats
])
def test_fp32_pipe_loaders_match_oracle(tcs, cx, sides, offset, loader):
    """Each loader of the FP32 pipe kernel (TMA, cp.async pairs, cp.async elements) gives the
    oracle's bits; the base offset forces the element loader on an even pitch.  (The plan names
    the loader of the pitch; the base is only known at launch.)"""
    import torch

    cfg = (3, "Star", "Row", "Jacobi", 2, cx, 2, 2, "None", 0)
    spec = G.spec_of(cfg, "f32")
    st = tcs.Stencil(spec)
    geom = spec.geometry(*sides)
    assert geom.grid[0] == sides[0]
    launch = tcs.Launch(block=(32 // cx, 4, 1), variant="pipe")
    assert st.plan(geom, launch).loader == loader
    a = np.random.default_rng(3).random(geom.shape).astype(np.float32)
    n = int(np.prod(geom.shape))
    bx = torch.zeros(n + 1, dtype=torch.float32, device="cuda")
    by = torch.zeros(n + 1, dtype=torch.float32, device="cuda")
    x = bx[offset:offset + n].view(geom.shape)
    y = by[offset:offset + n].view(geom.shape)
    x.copy_(torch.from_numpy(a))
    y.copy_(x)
    res = st.sweeps(geom, x, y, 3, launch)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    want = O.sweeps(O.make_spec(*cfg), a, 3, geom.right_offset)
    assert np.array_equal(res.cpu().numpy(), want)


@pytest.mark.parametrize("cfg, block, sides, precision, loader", [
    ((2, "Box", "Row", "Variable", 6, 8, 1, 1, "None", 0), (32, 1, 1), (300, 30), "f32", "cp.async pairs"),
    ((2, "Box", "Row", "Variable", 6, 8, 1, 1, "None", 0), (32, 1, 1), (300, 30), "f64", "cp.async"),
    ((3, "Star", "Row", "Jacobi", 2, 2, 2, 1, "Read", 16), (128, 1, 1), (290, 12, 10), "f64", "cp.async"),
])
def test_pipe_tiles_wider_than_a_tma_box(tcs, cfg, block, sides, precision, loader):
    """Single-grid pipe tiles wider than a 256-element TMA box stream their rows through cp.async
    and give the oracle's bits."""
    import torch

    spec = G.spec_of(cfg, precision)
    st = tcs.Stencil(spec)
    geom = spec.geometry(*sides)
    launch = tcs.Launch(block=block, variant="pipe")
    plan = st.plan(geom, launch)
    assert plan.loader == loader and plan.width > 256
    rng = np.random.default_rng(13)
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
