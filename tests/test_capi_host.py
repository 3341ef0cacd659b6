"""Host-side logic of libtcs.so (no GPU): exports, parameter checks, geometry, block shapes."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import threadcoarsenedstencilgenerator_b200 as tcs
from threadcoarsenedstencilgenerator_b200 import _lib
from threadcoarsenedstencilgenerator_b200.primes import block_shapes, prime_combinations

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_]+\**\s+\**(tcs_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 20
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for n in names:
        assert hasattr(lib, n), n
    # and the Python binding covers all of them
    assert set(names) <= set(_lib.SIGNATURES)


def test_abi_version():
    assert _lib.load().tcs_abi_version() == 2


@pytest.mark.parametrize("bad", [
    dict(dimension=4), dict(neighbourhood="Cross"), dict(orientation="Diag"), dict(coefficients="Mean"),
    dict(range=0), dict(cx=0), dict(alignment="Left"), dict(alignment="Read", cl_size=0),
])
def test_invalid_parameters_raise_invalid_value(bad):
    base = dict(dimension=2, neighbourhood="Box", orientation="Row", coefficients="Jacobi", range=1)
    base.update(bad)
    with pytest.raises(tcs.CudaErrorInvalidValue):
        tcs.StencilSpec(**base)


def test_stencil_size_and_flops():
    cases = [((2, "Box", 1), 9), ((2, "Star", 3), 13), ((3, "Box", 1), 27), ((3, "Star", 4), 25), ((2, "Box", 6), 169)]
    for (d, sh, r), S in cases:
        for coeff, flops in (("Jacobi", S), ("Variable", 2 * S - 1)):
            s = tcs.StencilSpec(dimension=d, neighbourhood=sh, range=r, coefficients=coeff)
            assert s.stencil_size == S and s.flops_per_update == flops


def test_geometry_matches_oracle_restatement():
    rng = np.random.default_rng(3)
    for _ in range(300):
        d = int(rng.integers(2, 4))
        r = int(rng.integers(1, 9))
        c = [int(v) for v in rng.integers(1, 9, size=3)]
        al = ["None", "Read", "Write"][int(rng.integers(0, 3))]
        cl = 0 if al == "None" else int(rng.choice([1, 2, 3, 4, 8, 16, 32]))
        n = [int(v) for v in rng.integers(2 * r, 300, size=3)]
        s = tcs.StencilSpec(dimension=d, range=r, cx=c[0], cy=c[1], cz=c[2], alignment=al, cl_size=cl)
        g = s.geometry(*n)
        o = O.geometry(O.make_spec(d, "Box", "Row", "Jacobi", r, c[0], c[1], c[2], al, cl), *n)
        assert g.grid == o.grid and g.elements == o.elements and g.threads == o.threads
        assert g.left_offset == o.left_offset and g.right_offset == o.right_offset and g.n_points == o.n_points
        if al != "None":
            assert g.grid[0] % cl == 0


def test_geometry_rejects_too_small_grid():
    s = tcs.StencilSpec(dimension=2, range=3)
    with pytest.raises(tcs.CudaErrorInvalidValue):
        s.geometry(5, 40)


def test_block_shape_enumeration_counts():
    # the reference's sweep at a 1024-thread limit (cuda/benchmark.cpp:223-318)
    assert len(block_shapes(2, 1024)) == 464
    assert len(block_shapes(3, 1024)) == 2723
    assert prime_combinations(96) == [1, 2, 4, 8, 16, 32, 3, 6, 12, 24, 48, 96]
    assert block_shapes(2, 64)[:3] == [(1, 32, 1), (2, 16, 1), (4, 8, 1)]


def test_create_without_device_reports_no_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(tcs.TcsError) as e:
        tcs.Stencil(tcs.StencilSpec())
    assert e.value.code == _lib.TCS_ERR_NO_DEVICE


def test_precompile_without_gpu(tmp_path, monkeypatch):
    monkeypatch.setenv("TCS_KCACHE", str(tmp_path))
    path = tcs.precompile(tcs.StencilSpec(dimension=3, neighbourhood="Star", coefficients="Variable", range=2,
                                          cx=2, cy=1, cz=2))
    assert Path(path).exists() and Path(path).stat().st_size > 1000


def test_ragged_geometry_keeps_the_whole_interior():
    from threadcoarsenedstencilgenerator_b200 import StencilSpec

    s = StencilSpec(dimension=3, neighbourhood="Star", coefficients="Variable", range=4, cx=2, cy=4, cz=3,
                    alignment="Read", cl_size=16)
    g = s.geometry(61, 47, 39, ragged=True)
    t = s.geometry(61, 47, 39)
    assert g.elements == (53, 39, 31) and t.elements == (52, 36, 30)
    assert g.threads == (27, 10, 11) and g.grid[1:] == (47, 39)
    assert g.grid[0] % 16 == 0 and g.grid[0] - g.right_offset == 61
    # multiples of the coarsening: identical to the reference geometry
    assert s.geometry(64, 48, 41, ragged=True) == s.geometry(64, 48, 41)


def test_entry_points_reject_null_handles_without_a_device():
    """Argument checks run before any device work: a NULL handle or buffer list is an invalid value."""
    lib = _lib.load()
    grid = _lib.U3(64, 64, 1)
    launch = _lib.CLaunch()
    rc = lib.tcs_sweep_host_jobs(None, grid, 0, ctypes.byref(launch), None, None, 1, 1, None, None, 1, None)
    assert rc == _lib.TCS_ERR_INVALID_VALUE
    assert "NULL" in lib.tcs_last_error().decode()
    res = ctypes.c_int()
    rc = lib.tcs_sweeps_tb2(None, grid, 0, None, None, 2, None, ctypes.byref(res))
    assert rc == _lib.TCS_ERR_INVALID_VALUE
    assert lib.tcs_self_test_wait(None, 2_000_000) == _lib.TCS_ERR_INVALID_VALUE
