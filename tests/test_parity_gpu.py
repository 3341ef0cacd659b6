"""GPU parity of the engine (C ABI through ctypes) with the reference and the oracle.

FP64 and FP32 results must be bit-identical (tolerance 0 ulp) to
  * the committed fixtures produced by the reference's own generated kernels,
  * the oracle on fresh seeded inputs,
  * the reference's generated kernels compiled for sm_100a and run on this GPU (oracle/_ref),
for both kernel variants and several block shapes; padding and border cells must stay untouched.
"""

import numpy as np
import pytest

import gpu_util as G
import oracle as O
from oracle import ref_configs
from make_golden import fixture_input, HERE as GOLDEN

pytestmark = pytest.mark.gpu

BLOCKS_2D = [(8, 4, 1), (32, 4, 1), (64, 1, 1), (16, 8, 1), (1, 32, 1), (32, 1, 1), (16, 1, 1)]
BLOCKS_3D = [(8, 4, 2), (32, 4, 1), (16, 4, 2), (8, 8, 1), (64, 2, 1), (16, 2, 1)]
PIPE_BLOCKS_2D = [(64, 1, 1), (32, 1, 1), (16, 1, 1)]
PIPE_BLOCKS_3D = [(32, 4, 1), (8, 8, 1), (16, 2, 1)]


@pytest.fixture(scope="module")
def tcs():
    import torch

    import threadcoarsenedstencilgenerator_b200 as t

    assert torch.cuda.is_available()
    return t


def _run_all_variants(tcs, cfg, a, g, n, mask, precision="f64"):
    spec = G.spec_of(cfg, precision)
    st = tcs.Stencil(spec)
    geom = spec.geometry(*((g.grid[0] - g.left_offset - g.right_offset,) + tuple(g.grid[1:])))
    assert geom.grid == tuple(g.grid)
    results = []
    blocks = BLOCKS_2D if cfg[0] == 2 else BLOCKS_3D
    for variant in ("direct", "march", "pipe"):
        for b in blocks:
            launch = tcs.Launch(block=b, variant=variant)
            try:
                st.plan(geom, launch)
            except tcs.UnsupportedLaunch:
                continue
            res, other, host = G.engine_sweeps(st, geom, a, n, launch, mask)
            results.append(((variant, b), res, host))
    assert st.device_status() == 0
    assert any(v == "march" for (v, _), _, _ in results), "no march shape ran for %s" % (cfg,)
    if not (cfg[0] == 2 and cfg[2] == "Column"):
        assert any(v == "pipe" for (v, _), _, _ in results), "no pipe shape ran for %s" % (cfg,)
    return geom, results


@pytest.mark.parametrize("cfg", ref_configs.PARITY, ids=ref_configs.key)
def test_engine_matches_reference_fixture(tcs, cfg):
    f = np.load(GOLDEN / ("%s.npz" % ref_configs.key(cfg)))
    spec, raw, g, a, mask = fixture_input(cfg, int(f["seed"]))
    want = f["out"]
    geom, results = _run_all_variants(tcs, cfg, a, g, int(f["nsweeps"]), mask)
    ls = geom.logical_slices()
    for (variant, b), res, host in results:
        assert np.array_equal(res[ls], want[ls]), "%s %s differs" % (variant, b)
        pad = np.ones(res.shape, bool)
        pad[ls] = False
        assert np.all(np.isnan(res[pad])), "padding written by %s %s" % (variant, b)


@pytest.mark.parametrize("cfg", ref_configs.PARITY, ids=ref_configs.key)
def test_reference_gpu_kernel_matches_oracle_and_engine(tcs, cfg):
    if not G.ref_lib_path(cfg).exists():
        pytest.skip("reference build not present")
    rng = np.random.default_rng(99)
    spec = O.make_spec(*cfg)
    n = (45, 38, 1) if cfg[0] == 2 else (29, 26, 23)
    g = O.geometry(spec, *n)
    a = rng.random((g.grid[1], g.grid[0]) if cfg[0] == 2 else (g.grid[2], g.grid[1], g.grid[0]))
    mask = None
    if cfg[3] == "Variable":
        m = rng.standard_normal(O.stencil_size(spec))
        mask = m / m.sum()
    ref = G.reference_sweeps(cfg, g.grid, g.threads, g.right_offset, a, 2, mask)
    orc = O.sweeps(spec, a, 2, g.right_offset, mask)
    ls = (slice(None),) * (cfg[0] - 1) + (slice(g.left_offset, g.grid[0] - g.right_offset),)
    assert np.array_equal(ref[ls], orc[ls]), "oracle differs from the reference kernel on the GPU"
    geom, results = _run_all_variants(tcs, cfg, a, g, 2, mask)
    for (variant, b), res, host in results:
        assert np.array_equal(res[ls], ref[ls]), "%s %s differs from the reference kernel" % (variant, b)


@pytest.mark.parametrize("cfg", ref_configs.PARITY[::2], ids=ref_configs.key)
def test_engine_fp32_matches_oracle(tcs, cfg):
    rng = np.random.default_rng(5)
    spec = O.make_spec(*cfg)
    n = (50, 41, 1) if cfg[0] == 2 else (30, 27, 25)
    g = O.geometry(spec, *n)
    a = rng.random((g.grid[1], g.grid[0]) if cfg[0] == 2 else (g.grid[2], g.grid[1], g.grid[0])).astype(np.float32)
    mask = rng.standard_normal(O.stencil_size(spec)) if cfg[3] == "Variable" else None
    want = O.sweeps(spec, a, 3, g.right_offset, mask)
    geom, results = _run_all_variants(tcs, cfg, a, g, 3, mask, precision="f32")
    ls = geom.logical_slices()
    for (variant, b), res, host in results:
        assert np.array_equal(res[ls], want[ls]), "%s %s differs" % (variant, b)


def test_init_kernel_matches_reference_pattern(tcs):
    import torch

    for cfg in [(2, "Box", "Row", "Jacobi", 2, 1, 1, 1, "Write", 8), (3, "Star", "Row", "Jacobi", 1, 1, 1, 1, "None", 0),
                (3, "Box", "Column", "Variable", 2, 1, 2, 1, "Read", 16)]:
        spec = G.spec_of(cfg)
        st = tcs.Stencil(spec)
        geom = spec.geometry(37, 23, 19)
        d = torch.full(geom.shape, float("nan"), dtype=torch.float64, device="cuda")
        block = (32, 16, 1) if cfg[0] == 2 else (16, 16, 4)
        gb = tuple(-(-geom.grid[i] // block[i]) for i in range(3))
        st.launch_init(geom.grid, block, gb, d, geom.right_offset)
        want = O.init_pattern(O.make_spec(*cfg), geom.grid, geom.right_offset)
        got = d.cpu().numpy()
        assert np.array_equal(np.isnan(got), np.isnan(want)) and np.array_equal(got[~np.isnan(got)], want[~np.isnan(want)])


def test_benchmark_update_grid_dropin(tcs):
    import torch

    cfg = (2, "Star", "Row", "Variable", 2, 2, 2, 1, "Read", 16)
    spec = G.spec_of(cfg)
    lug = tcs.LaunchUpdateGrid(spec)
    geom = spec.geometry(130, 90)
    rng = np.random.default_rng(2)
    a = rng.random(geom.shape)
    m = rng.standard_normal(spec.stencil_size)
    lug.copyMask(m, spec.stencil_size)
    d0 = torch.from_numpy(a).cuda()
    d1 = d0.clone()
    block = (32, 4, 1)
    gb = tuple(-(-geom.threads[i] // block[i]) for i in range(3))
    durations = lug.benchmarkUpdateGrid("Variable", "Star", 2, 2, "Read", 0.0, geom.grid, block, gb, d0, d1,
                                        geom.right_offset)
    assert len(durations) == 1 and durations[0] > 0
    want = O.sweep(O.make_spec(*cfg), a, geom.right_offset, m)
    assert np.array_equal(d1.cpu().numpy()[geom.logical_slices()], want[geom.logical_slices()])
    durations = lug.benchmarkUpdateGrid("Variable", "Star", 2, 2, "Read", 0.05, geom.grid, block, gb, d0, d1,
                                        geom.right_offset)
    assert len(durations) >= 3 and len(durations) + 1 & len(durations) == 0  # 2^k - 1 launches
    with pytest.raises(tcs.CudaErrorInvalidValue):
        lug.benchmarkUpdateGrid("Jacobi", "Star", 2, 2, "Read", 0.0, geom.grid, block, gb, d0, d1, geom.right_offset)
    with pytest.raises(tcs.CudaErrorInvalidValue):
        lug.benchmarkUpdateGrid("Variable", "Star", 3, 2, "Read", 0.0, geom.grid, block, gb, d0, d1, geom.right_offset)
    assert lug.maxPotentialBlockSize() >= 32


@pytest.mark.parametrize("block", [(128, 1, 1), (32, 4, 1), (64, 2, 1)])
def test_benchmark_update_grid_dropin_each_variant(tcs, block):
    """The drop-in with the engine's default choice for each block shape (pipe / march)."""
    import torch

    cfg = (2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0)
    spec = G.spec_of(cfg)
    lug = tcs.LaunchUpdateGrid(spec)
    geom = spec.geometry(1024, 1024)
    a = np.random.default_rng(4).random(geom.shape)
    d0 = torch.from_numpy(a).cuda()
    d1 = d0.clone()
    gb = tuple(-(-geom.threads[i] // block[i]) for i in range(3))
    durations = lug.benchmarkUpdateGrid("Jacobi", "Box", 1, 2, "None", 0.0, geom.grid, block, gb, d0, d1, 0)
    assert len(durations) == 1
    want = O.sweep(O.make_spec(*cfg), a)
    assert np.array_equal(d1.cpu().numpy(), want)
    durations = lug.benchmarkUpdateGrid("Jacobi", "Box", 1, 2, "None", 0.02, geom.grid, block, gb, d0, d1, 0)
    assert len(durations) >= 3


def test_full_size_2d_box_jacobi_against_oracle(tcs):
    """The 4096^2 Box Jacobi r1 workload: 4 sweeps, bit-identical with the oracle."""
    import torch

    cfg = (2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0)
    spec = G.spec_of(cfg)
    st = tcs.Stencil(spec)
    geom = spec.geometry(4096, 4096)
    rng = np.random.default_rng(0)
    a = rng.random(geom.shape)
    want = O.sweeps(O.make_spec(*cfg), a, 4, 0, None, cpu_threads=0)
    for launch in (tcs.Launch(block=(64, 4, 1), variant="march"), tcs.Launch(block=(128, 1, 1), variant="direct")):
        x = torch.from_numpy(a).cuda()
        y = x.clone()
        res = st.sweeps(geom, x, y, 4, launch)
        assert np.array_equal(res.cpu().numpy(), want)
