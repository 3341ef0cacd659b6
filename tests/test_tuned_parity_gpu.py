"""Every launch the benchmark times, bit for bit against the oracle on the GPU.

bench.py runs each workload with its tuned launch (tuned.json: coarsening, kernel variant, block,
planes per ring chunk, chunks in flight).  These tests run exactly those instantiations -- the
workload's parameter set with the tuned coarsening, the tuned Launch -- and require the result to
equal the oracle's at 0 ulp:

  * on a mid-size grid with at least three tiles of the launch along every tiled axis and ragged
    last tiles (partial tiles in x and y, work items of the persistent kernels split across tile
    boundaries), for several sweeps;
  * on the workload's full grid for two sweeps (the oracle's OpenMP loop, same per-output order);
  * for the batch workload, every grid of the 64-grid batch, FP64 and FP32, with the tuned batch
    launches.

The planner is asked to confirm the variant and loader, so a change of tuned.json that the planner
would silently turn into another kernel fails here.
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


def _ospec(spec):
    return O.make_spec(spec.dimension, spec.neighbourhood, spec.orientation, spec.coefficients, spec.range, spec.cx,
                       spec.cy, spec.cz, spec.alignment, spec.cl_size)


def _mid_grid(spec, plan):
    """Raw grid extents with >= 3 tiles of the plan per tiled axis plus a ragged remainder."""
    R = spec.range
    tx = plan.block[0] * spec.cx
    if spec.dimension == 2:
        ty = plan.block[1] * spec.cy
        rows = 3 * ty + 5 * spec.cy + R if plan.variant == "direct" else 3 * 64 + 11
        return (2 * R + 3 * tx + 5 * spec.cx + 3, 2 * R + rows, 1)
    ty = plan.block[1] * spec.cy
    return (2 * R + 3 * tx + 5 * spec.cx + 3, 2 * R + 3 * ty + 3 * spec.cy + 1, 2 * R + 37)


def _run(tcs, spec, launch, geom, a, mask, n):
    import torch

    st = tcs.Stencil(spec)
    if mask is not None:
        st.copy_mask(mask)
    x = torch.from_numpy(a).cuda()
    y = x.clone()
    res = st.sweeps(geom, x, y, n, launch)
    torch.cuda.synchronize()
    assert st.device_status() == 0
    out = res.cpu().numpy()
    st.close()
    return out


def _workload_names():
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    return sorted(WORKLOADS)


@pytest.mark.parametrize("name", _workload_names())
def test_tuned_launch_mid_grid_matches_oracle(tcs, name):
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    w = WORKLOADS[name]
    spec = w.tuned_spec()
    launch = w.tuned_launch()
    st = tcs.Stencil(spec)
    full = spec.geometry(*w.grid)
    plan = st.plan(full, launch)
    assert plan.variant == launch.variant
    geom = spec.geometry(*_mid_grid(spec, plan))
    mplan = st.plan(geom, launch)
    assert (mplan.variant, mplan.loader, mplan.chunk) == (plan.variant, plan.loader, plan.chunk)
    st.close()
    tiles_x = -(-geom.elements[0] // (plan.block[0] * spec.cx))
    assert tiles_x >= 3 and geom.elements[0] % (plan.block[0] * spec.cx) != 0
    if spec.dimension == 3:
        assert -(-geom.elements[1] // (plan.block[1] * spec.cy)) >= 3
    a = w.make_input(geom)
    mask = w.make_mask()
    n = 5
    got = _run(tcs, spec, launch, geom, a, mask, n)
    want = O.sweeps(_ospec(spec), a, n, geom.right_offset, mask)
    assert np.array_equal(got, want), "max |diff| %g" % float(np.abs(got - want).max())


@pytest.mark.parametrize("name", _workload_names())
def test_tuned_launch_full_grid_matches_oracle(tcs, name):
    """The benchmarked instantiation on the workload's own grid and data, two sweeps."""
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    w = WORKLOADS[name]
    spec = w.tuned_spec()
    launch = w.tuned_launch()
    geom = spec.geometry(*w.grid)
    a = w.make_input(geom)
    mask = w.make_mask()
    got = _run(tcs, spec, launch, geom, a, mask, 2)
    want = O.sweeps(_ospec(spec), a, 2, geom.right_offset, mask, cpu_threads=0)
    assert np.array_equal(got, want), "max |diff| %g" % float(np.abs(got - want).max())


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_tuned_batch_launch_every_grid_matches_oracle(tcs, precision):
    """All 64 grids of the batch workload with its tuned launch (per precision), 2 sweeps in one
    captured graph, each grid against the oracle."""
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
    xs = [torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in arrs]
    ys = [x.clone() for x in xs]
    bt = BatchedSweeps(st, geoms, xs, ys, launch)
    assert tuple(bt.plan().block) == tuple(launch.block)
    bt.capture(2)
    res = bt.replay()
    torch.cuda.synchronize()
    assert st.device_status() == 0
    ospec = _ospec(spec)
    for i, (g, v, r) in enumerate(zip(geoms, arrs, res)):
        want = O.sweeps(ospec, v, 2, g.right_offset, None, cpu_threads=0)
        assert np.array_equal(r.cpu().numpy(), want), "grid %d %s" % (i, g.grid)
    bt.close()
