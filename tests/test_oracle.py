"""The CPU oracle, pinned against the reference's own kernels.

The fixtures in tests/golden/ were produced by the reference's generated kernels
(tests/golden/make_golden.py); the oracle must reproduce them bit for bit.  Further self-made
known-answer tests follow the reference's semantics (constant and linear fields, the init pattern).
"""

import numpy as np
import pytest

import oracle as O
from oracle import ref_configs
from make_golden import fixture_input, HERE as GOLDEN


@pytest.mark.parametrize("cfg", ref_configs.PARITY, ids=ref_configs.key)
def test_oracle_matches_reference_fixture(cfg):
    f = np.load(GOLDEN / ("%s.npz" % ref_configs.key(cfg)))
    spec, raw, g, a, mask = fixture_input(cfg, int(f["seed"]))
    assert tuple(int(v) for v in f["raw"]) == tuple(raw)
    out = O.sweeps(spec, a, int(f["nsweeps"]), g.right_offset, mask)
    assert np.array_equal(out, f["out"])


@pytest.mark.parametrize("cfg", ref_configs.EXTRA, ids=ref_configs.key)
def test_oracle_matches_reference_fixture_long_ranges(cfg):
    """Ranges 5-8, 3D Box beyond range 1 and wider coarsening: the oracle against fixtures from
    the reference's generated kernels (host build), bit for bit, and its OpenMP loop likewise."""
    f = np.load(GOLDEN / ("%s.npz" % ref_configs.key(cfg)))
    assert str(f["source"]) == "host-shim"
    spec, raw, g, a, mask = fixture_input(cfg, int(f["seed"]))
    assert tuple(int(v) for v in f["raw"]) == tuple(raw)
    assert np.array_equal(O.sweeps(spec, a, int(f["nsweeps"]), g.right_offset, mask), f["out"])
    assert np.array_equal(O.sweeps(spec, a, int(f["nsweeps"]), g.right_offset, mask, cpu_threads=4), f["out"])


@pytest.mark.parametrize("cfg", ref_configs.PARITY, ids=ref_configs.key)
def test_openmp_baseline_is_bit_identical(cfg):
    f = np.load(GOLDEN / ("%s.npz" % ref_configs.key(cfg)))
    spec, raw, g, a, mask = fixture_input(cfg, int(f["seed"]))
    out = O.sweeps(spec, a, int(f["nsweeps"]), g.right_offset, mask, cpu_threads=4)
    assert np.array_equal(out, f["out"])


def test_term_order_independent_of_coarsening():
    rng = np.random.default_rng(7)
    for dim in (2, 3):
        for sh in ("Box", "Star"):
            for o in ("Row", "Column"):
                for r in (1, 2, 3):
                    base = O.make_spec(dim, sh, o, "Variable", r, 1, 1, 1)
                    n = (29, 23, 19) if dim == 3 else (41, 37, 1)
                    g = O.geometry(base, *n)
                    shape = (g.grid[1], g.grid[0]) if dim == 2 else (g.grid[2], g.grid[1], g.grid[0])
                    a = rng.random(shape)
                    m = rng.standard_normal(O.stencil_size(base))
                    ref = O.sweep(base, a, 0, m)
                    for c in ((2, 1, 1), (1, 3, 1), (3, 2, 2)):
                        s = O.make_spec(dim, sh, o, "Variable", r, *c)
                        gg = O.geometry(s, *n)
                        # same buffer: only the truncated interior differs
                        out = O.sweep(s, a[tuple(slice(0, k) for k in a.shape)], 0, m)
                        sl = tuple(slice(r, r + e) for e in reversed(gg.elements[:dim]))
                        assert np.array_equal(out[sl], ref[sl])


def test_constant_field_stays_constant_jacobi():
    for dim in (2, 3):
        for sh in ("Box", "Star"):
            s = O.make_spec(dim, sh, "Row", "Jacobi", 2, 1, 1, 1)
            n = (21, 17, 13) if dim == 3 else (33, 31, 1)
            g = O.geometry(s, *n)
            shape = (g.grid[1], g.grid[0]) if dim == 2 else (g.grid[2], g.grid[1], g.grid[0])
            a = np.full(shape, 0.5)
            out = O.sweeps(s, a, 4)
            # 0.5 * S summed exactly, times fl(1/S): within one rounding of 0.5
            assert np.allclose(out, 0.5, rtol=0, atol=1e-15)


def test_linear_field_reproduced_by_symmetric_mask():
    s = O.make_spec(2, "Box", "Column", "Variable", 2, 2, 2)
    g = O.geometry(s, 30, 26)
    y, x = np.mgrid[0:g.grid[1], 0:g.grid[0]].astype(np.float64)
    a = 0.25 * x + 0.5 * y
    S = O.stencil_size(s)
    m = np.full(S, 1.0 / S)
    out = O.sweep(s, a, 0, m)
    sl = (slice(2, 2 + g.elements[1]), slice(2, 2 + g.elements[0]))
    assert np.allclose(out[sl], a[sl], rtol=1e-13, atol=1e-12)


def test_hand_computed_5x5_star():
    s = O.make_spec(2, "Star", "Row", "Variable", 1, 1, 1)
    a = np.arange(25, dtype=np.float64).reshape(5, 5)
    m = np.array([1.0, 2.0, 3.0, 4.0, 5.0])  # up, left, centre, right, down
    out = O.sweep(s, a, 0, m)
    # centre (2,2) = 1*a[1,2] + 2*a[2,1] + 3*a[2,2] + 4*a[2,3] + 5*a[3,2]
    assert out[2, 2] == 1 * 7 + 2 * 11 + 3 * 12 + 4 * 13 + 5 * 17
    assert out[0, 0] == a[0, 0] and out[4, 4] == a[4, 4]


def test_init_pattern_2d_and_3d():
    s = O.make_spec(2, "Box", "Row", "Jacobi", 2, 1, 1, 1, "Write", 8)
    g = O.geometry(s, 20, 10)
    a = O.init_pattern(s, g.grid, g.right_offset)
    lo = g.left_offset
    assert np.all(np.isnan(a[:, :lo]))                       # left padding untouched
    assert np.all(a[:, lo:lo + 2] == 1.0) and np.all(a[:2, lo:g.grid[0] - g.right_offset] == 1.0)
    assert np.all(a[2:, lo + 2:g.grid[0] - g.right_offset] == 0.0)
    s3 = O.make_spec(3, "Star", "Row", "Jacobi", 1, 1, 1, 1)
    g3 = O.geometry(s3, 6, 5, 4)
    b = O.init_pattern(s3, g3.grid, 0)
    idx = np.arange(b.size).reshape(b.shape)
    border = np.zeros(b.shape, bool)
    border[0] = True
    border[:, 0] = True
    border[:, :, 0] = True
    assert np.all(b[border] == np.where(idx[border] % 2 == 0, 0.75, 0.25))
    assert np.all(b[~border] == 0.0)


def test_geometry_rules():
    s = O.make_spec(3, "Star", "Row", "Variable", 4, 1, 1, 1, "Read", 16)
    g = O.geometry(s, 512, 512, 512)
    assert g.grid == (512, 512, 512) and g.right_offset == 0 and g.elements == (504, 504, 504)
    s = O.make_spec(2, "Box", "Row", "Jacobi", 1, 3, 2, 1, "Write", 16)
    g = O.geometry(s, 100, 50)
    # truncation: 100 - (98 % 3) = 98; Write: left = 16 - 1 = 15; 98+15=113 -> right 15 -> 128
    assert g.left_offset == 15 and g.right_offset == 15 and g.grid[0] == 128 and g.grid[1] == 50 - (48 % 2)
