"""Host-buffer job runner (tcs_sweep_host_jobs) against the oracle.

Every job uploads its own host grid, runs n sweeps and downloads the result; jobs rotate over
device slots whose streams overlap one another.  Each job's result must equal n oracle sweeps of
its input bit for bit, whatever the slot count (a race between slots would mix grids).
"""

import numpy as np
import pytest

import gpu_util as G
import oracle as O

pytestmark = pytest.mark.gpu

CASES = [
    ((3, "Star", "Row", "Variable", 2, 2, 2, 1, "Read", 16), "f64", (45, 30, 24), 3, False),
    ((2, "Box", "Row", "Jacobi", 1, 2, 2, 1, "None", 0), "f32", (130, 70), 2, False),
    ((3, "Box", "Row", "Variable", 1, 2, 4, 1, "None", 0), "f64", (37, 23, 19), 2, True),
]


@pytest.fixture(scope="module")
def tcs():
    import threadcoarsenedstencilgenerator_b200 as t

    return t


@pytest.mark.parametrize("slots", [1, 2, 3])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "%dD_%s_%s%s" % (c[0][0], c[0][1], c[1],
                                                                         "_ragged" if c[4] else ""))
def test_host_jobs_match_oracle(tcs, case, slots):
    import torch

    cfg, prec, sides, n, ragged = case
    spec = G.spec_of(cfg, prec)
    st = tcs.Stencil(spec)
    geom = spec.geometry(*sides, ragged=ragged)
    dt = np.float64 if prec == "f64" else np.float32
    rng = np.random.default_rng(slots)
    mask = rng.standard_normal(spec.stencil_size) if cfg[3] == "Variable" else None
    if mask is not None:
        st.copy_mask(mask)
    njobs = 5
    ins = [rng.uniform(-1, 1, geom.shape).astype(dt) for _ in range(njobs)]
    host_in = [torch.from_numpy(a).pin_memory() for a in ins]
    host_out = [torch.full(geom.shape, float("nan"), dtype=host_in[0].dtype).pin_memory() for _ in range(njobs)]
    ms = st.sweep_host_jobs(geom, host_in, host_out, n, tcs.Launch(block=(32, 4, 1)), slots=slots)
    assert ms > 0
    assert st.device_status() == 0
    # the per-point term order does not depend on the coarsening, so a ragged grid (its partial
    # tiles swept with coarsening 1) equals the coarsening-1 oracle
    ospec = O.make_spec(*(cfg[:5] + ((1, 1, 1) if ragged else cfg[5:8]) + cfg[8:]))
    for a, r in zip(ins, host_out):
        assert np.array_equal(r.numpy(), O.sweeps(ospec, a, n, geom.right_offset, mask))


def test_host_jobs_reuse_outputs_within_a_slot(tcs):
    """Jobs j and j + slots may share a host output: the later download lands last."""
    import torch

    cfg = (3, "Star", "Row", "Jacobi", 1, 1, 1, 1, "None", 0)
    spec = G.spec_of(cfg)
    st = tcs.Stencil(spec)
    geom = spec.geometry(20, 18, 16)
    rng = np.random.default_rng(4)
    ins = [rng.random(geom.shape) for _ in range(4)]
    host_in = [torch.from_numpy(a) for a in ins]
    outs = [torch.empty(geom.shape, dtype=torch.float64) for _ in range(2)]
    st.sweep_host_jobs(geom, host_in, [outs[j % 2] for j in range(4)], 2, slots=2)
    ospec = O.make_spec(*cfg)
    assert np.array_equal(outs[0].numpy(), O.sweeps(ospec, ins[2], 2, geom.right_offset))
    assert np.array_equal(outs[1].numpy(), O.sweeps(ospec, ins[3], 2, geom.right_offset))


def test_host_jobs_reject_bad_arguments(tcs):
    import torch

    spec = G.spec_of((3, "Star", "Row", "Jacobi", 1, 1, 1, 1, "None", 0))
    st = tcs.Stencil(spec)
    geom = spec.geometry(20, 18, 16)
    a = torch.zeros(geom.shape, dtype=torch.float64)
    o1, o2 = torch.zeros_like(a), torch.zeros_like(a)
    with pytest.raises(ValueError):
        st.sweep_host_jobs(geom, [a, a], [o1], 1)
    with pytest.raises(ValueError):  # jobs 0 and 1 run on different slots
        st.sweep_host_jobs(geom, [a, a], [o1, o1], 1, slots=2)
    with pytest.raises(ValueError):  # output aliases an input
        st.sweep_host_jobs(geom, [a], [a], 1)
    with pytest.raises(ValueError):  # wrong dtype
        st.sweep_host_jobs(geom, [a.float()], [o2.float()], 1)
    with pytest.raises(ValueError):  # device tensor
        st.sweep_host_jobs(geom, [a.cuda()], [o2], 1)
    st.sweep_host_jobs(geom, [a], [o2], 1, slots=2)  # more slots than jobs: one slot used
