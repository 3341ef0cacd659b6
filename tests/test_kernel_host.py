"""The engine's kernel arithmetic and addressing, checked on the CPU.

* tcs_tile.cuh (the per-thread arithmetic every sweep kernel runs) is compiled for the host and
  compared bit for bit with the reference fixtures and with the oracle on random parameter sets.
* The march kernel's TMA/ring addressing is replayed by tests/march_model.py for many shapes.
"""

import numpy as np
import pytest

import host_tile
import march_model
import pipe_model
import oracle as O
from oracle import ref_configs
from make_golden import fixture_input, HERE as GOLDEN


@pytest.mark.parametrize("cfg", ref_configs.PARITY + ref_configs.EXTRA, ids=ref_configs.key)
def test_kernel_arithmetic_matches_reference_fixture(cfg):
    f = np.load(GOLDEN / ("%s.npz" % ref_configs.key(cfg)))
    spec, raw, g, a, mask = fixture_input(cfg, int(f["seed"]))
    out = host_tile.sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, int(f["nsweeps"]), mask)
    assert np.array_equal(out, f["out"])


def _random_cfgs(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        d = int(rng.integers(2, 4))
        r = int(rng.integers(1, 4 if d == 3 else 6))
        c = [int(v) for v in rng.integers(1, 4, size=3)]
        al = ["None", "Read", "Write"][int(rng.integers(0, 3))]
        cl = 0 if al == "None" else int(rng.choice([4, 8, 16]))
        out.append((d, ["Box", "Star"][int(rng.integers(0, 2))], ["Row", "Column"][int(rng.integers(0, 2))],
                    ["Jacobi", "Variable"][int(rng.integers(0, 2))], r, c[0], c[1], c[2] if d == 3 else 1, al, cl))
    return out


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("cfg", _random_cfgs(8, 11), ids=ref_configs.key)
def test_kernel_arithmetic_matches_oracle_random(cfg, precision):
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec = O.make_spec(*cfg)
    n = (20 + 2 * r, 17 + 2 * r, 13 + 2 * r)
    g = O.geometry(spec, *n)
    rng = np.random.default_rng(5)
    shape = (g.grid[1], g.grid[0]) if d == 2 else (g.grid[2], g.grid[1], g.grid[0])
    dt = np.float64 if precision == "f64" else np.float32
    a = rng.random(shape).astype(dt)
    mask = rng.standard_normal(O.stencil_size(spec)) if c == "Variable" else None
    want = O.sweeps(spec, a, 2, g.right_offset, mask)
    got = host_tile.sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, 2, mask, precision)
    assert np.array_equal(got, want)


MARCH_CASES = [
    (2, "Box", 1, (1, 1, 1), (32, 4, 1), (40, 30, 1), "None", 0),
    (2, "Box", 1, (1, 1, 1), (64, 1, 1), (70, 11, 1), "None", 0),
    (2, "Star", 3, (2, 1, 1), (16, 2, 1), (61, 45, 1), "Write", 8),
    (2, "Box", 2, (3, 2, 1), (8, 4, 1), (53, 40, 1), "Read", 16),
    (2, "Box", 6, (2, 2, 1), (16, 2, 1), (60, 33, 1), "None", 0),
    (2, "Star", 1, (1, 1, 1), (1, 32, 1), (12, 80, 1), "Write", 16),
    # shapes whose natural chunk size is not a multiple of 128 bytes (TMA destination rule)
    (2, "Box", 1, (1, 1, 1), (128, 2, 1), (300, 20, 1), "None", 0),
    (2, "Box", 2, (2, 3, 1), (8, 4, 1), (37, 29, 1), "None", 0),
    (3, "Star", 4, (1, 1, 1), (32, 4, 1), (40, 30, 28), "Read", 16),
    (3, "Star", 4, (2, 2, 1), (16, 4, 1), (44, 29, 21), "Read", 16),
    (3, "Star", 2, (2, 2, 2), (8, 4, 2), (31, 29, 27), "None", 0),
    (3, "Box", 1, (1, 3, 1), (16, 2, 3), (35, 26, 22), "Write", 16),
    (3, "Box", 2, (1, 1, 2), (8, 8, 1), (22, 21, 20), "None", 0),
]


@pytest.mark.parametrize("case", MARCH_CASES, ids=lambda c: "%dD_%s_r%d_c%s_b%s" % (c[0], c[1], c[2], c[3], c[4]))
@pytest.mark.parametrize("es", [8, 4])
def test_march_addressing_model(case, es):
    d, sh, r, c, blk, n, al, cl = case
    spec = O.make_spec(d, sh, "Row", "Jacobi", r, c[0], c[1], c[2], al, cl)
    g = O.geometry(spec, *n)
    grid = g.grid
    for seg in (0, 1, 3):
        for depth in (0, 1, 3):
            cnt = march_model.simulate(d, sh, r, c, blk, grid, g.left_offset, g.right_offset, al != "None", es=es,
                                       segments=seg, depth=depth, num_sms=5)
            assert cnt is None or cnt > 0


PIPE_CFGS = [c for c in ref_configs.PARITY + ref_configs.EXTRA if not (c[0] == 2 and c[2] == "Column")]


@pytest.mark.parametrize("cfg", PIPE_CFGS, ids=ref_configs.key)
def test_pipe_arithmetic_matches_reference_fixture(cfg):
    f = np.load(GOLDEN / ("%s.npz" % ref_configs.key(cfg)))
    spec, raw, g, a, mask = fixture_input(cfg, int(f["seed"]))
    for piece, unroll in ((1 << 30, 0), (5, 1), (7, 2), (4, 3)):
        if unroll > 2 * cfg[4] + 1:
            continue
        out = host_tile.pipe_sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, int(f["nsweeps"]), mask,
                                    piece=piece, unroll=unroll)
        assert np.array_equal(out, f["out"])


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("cfg", [c for c in _random_cfgs(10, 17) if not (c[0] == 2 and c[2] == "Column")],
                         ids=ref_configs.key)
def test_pipe_arithmetic_matches_oracle_random(cfg, precision):
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec = O.make_spec(*cfg)
    g = O.geometry(spec, 20 + 2 * r, 17 + 2 * r, 13 + 2 * r)
    rng = np.random.default_rng(8)
    shape = (g.grid[1], g.grid[0]) if d == 2 else (g.grid[2], g.grid[1], g.grid[0])
    a = rng.random(shape).astype(np.float64 if precision == "f64" else np.float32)
    mask = rng.standard_normal(O.stencil_size(spec)) if c == "Variable" else None
    want = O.sweeps(spec, a, 2, g.right_offset, mask)
    got = host_tile.pipe_sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, 2, mask, precision, piece=6,
                                unroll=1 + (r % 2))
    assert np.array_equal(got, want)


RING_CFGS = [
    (3, "Star", "Row", "Variable", 4, 2, 4, 1, "Read", 16),
    (3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16),
    (3, "Star", "Row", "Jacobi", 1, 1, 1, 1, "None", 0),
    (3, "Star", "Row", "Variable", 2, 2, 2, 1, "Write", 8),
    (3, "Star", "Row", "Jacobi", 3, 1, 4, 1, "None", 0),
    (3, "Star", "Row", "Variable", 5, 2, 1, 1, "Read", 16),
]


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("cfg", RING_CFGS, ids=ref_configs.key)
def test_pipe_ring_form_matches_oracle(cfg, precision):
    """The ring form (own values and finished crosses kept in two R-entry rings instead of 2R+1
    output planes in registers) is bit-identical to the oracle, with pieces restarting the rings
    from stale contents."""
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec = O.make_spec(*cfg)
    g = O.geometry(spec, 19 + 2 * r, 15 + 2 * r, 14 + 2 * r)
    rng = np.random.default_rng(9)
    a = rng.random((g.grid[2], g.grid[1], g.grid[0])).astype(np.float64 if precision == "f64" else np.float32)
    mask = rng.standard_normal(O.stencil_size(spec)) if c == "Variable" else None
    want = O.sweeps(spec, a, 2, g.right_offset, mask)
    for piece in (1 << 30, 5, 1):
        got = host_tile.pipe_ring_sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, 2, mask, precision,
                                         piece=piece)
        assert np.array_equal(got, want), piece


PAIR_CFGS = [
    (2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0),
    (2, "Box", "Row", "Variable", 3, 8, 1, 1, "Read", 16),
    (2, "Box", "Row", "Jacobi", 1, 2, 1, 1, "Write", 8),
    (3, "Box", "Row", "Jacobi", 1, 2, 2, 1, "None", 0),
    (3, "Box", "Row", "Variable", 2, 2, 1, 1, "Write", 16),
    (3, "Box", "Row", "Variable", 1, 4, 2, 1, "Read", 8),
]


@pytest.mark.parametrize("cfg", PAIR_CFGS, ids=ref_configs.key)
def test_pipe_packed_fp32_pairs_match_oracle(cfg):
    """FP32 Box Row stencils with an even x coarsening take the packed-pair path (two outputs per
    f32x2 instruction, lane by lane the scalar rounding): bit-identical to the float oracle."""
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec = O.make_spec(*cfg)
    g = O.geometry(spec, 23 + 2 * r + 3 * cx, 19 + 2 * r, 11 + 2 * r)
    rng = np.random.default_rng(21)
    shape = (g.grid[1], g.grid[0]) if d == 2 else (g.grid[2], g.grid[1], g.grid[0])
    a = rng.uniform(-1, 1, shape).astype(np.float32)
    mask = rng.standard_normal(O.stencil_size(spec)) if c == "Variable" else None
    want = O.sweeps(spec, a, 3, g.right_offset, mask)
    for piece, unroll in ((1 << 30, 1), (5, 2), (4, 3)):
        got = host_tile.pipe_sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, 3, mask, "f32", piece=piece,
                                    unroll=unroll)
        assert np.array_equal(got, want)


COMP_PAIR_CFGS = [
    (2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0),
    (2, "Box", "Row", "Jacobi", 3, 2, 1, 1, "None", 0),
    (3, "Box", "Row", "Variable", 2, 2, 2, 1, "Read", 16),
]


@pytest.mark.parametrize("cfg", COMP_PAIR_CFGS, ids=ref_configs.key)
def test_pipe_compensated_rows_within_bound(cfg):
    """The pipelined kernel's compensated FP32 form (packed Box path): each footprint row's 2R+1
    terms are summed with plain FMAs, the row partials with two-sum.  Per point, against the float64
    oracle on the same FP32 inputs and FP32-rounded mask:
        |f32c - exact| <= 3u |exact| + (2R + 2) u sum |mask| |in|,   u = 2^-24,
    and plain FP32 (bound (S + 1) u sum |mask| |in|) does worse on the long stencil."""
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec = O.make_spec(*cfg)
    g = O.geometry(spec, 21 + 2 * r + 3 * cx, 17 + 2 * r, 9 + 2 * r)
    rng = np.random.default_rng(31)
    shape = (g.grid[1], g.grid[0]) if d == 2 else (g.grid[2], g.grid[1], g.grid[0])
    a = rng.uniform(-1, 1, shape).astype(np.float32)
    S = O.stencil_size(spec)
    mask = rng.standard_normal(S) / S if c == "Variable" else None
    got = host_tile.pipe_sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, 1, mask, "f32c", piece=5,
                                unroll=2).astype(np.float64)
    plain = host_tile.pipe_sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, 1, mask, "f32", piece=5,
                                  unroll=2).astype(np.float64)
    m32 = None if mask is None else mask.astype(np.float32).astype(np.float64)
    exact = O.sweep(spec, a.astype(np.float64), g.right_offset, m32)
    absm = None if m32 is None else np.abs(m32)
    mag = O.sweep(spec, np.abs(a.astype(np.float64)), g.right_offset, absm)
    u = 2.0 ** -24
    if c == "Jacobi":  # the oracle scales by the double 1/S; the FP32 sweeps by fl32(1/S)
        exact = exact * (np.float64(np.float32(1.0 / S)) * S)
        mag = mag * (np.float64(np.float32(1.0 / S)) * S)
    bound = 3 * u * np.abs(exact) + (2 * r + 2) * u * mag
    err = np.abs(got - exact)
    assert np.all(err <= bound), float((err / bound).max())
    if c == "Variable":
        assert err.max() < np.abs(plain - exact).max()


PIPE_CASES = [
    (2, "Box", 1, (1, 1, 1), (32, 1, 1), (70, 23, 1), "None", 0),
    (2, "Box", 6, (2, 1, 1), (16, 1, 1), (80, 40, 1), "None", 0),
    (2, "Star", 3, (2, 1, 1), (8, 1, 1), (61, 45, 1), "Write", 8),
    (2, "Star", 1, (1, 1, 1), (64, 1, 1), (37, 29, 1), "Read", 16),
    (3, "Star", 4, (2, 2, 1), (8, 4, 1), (44, 29, 21), "Read", 16),
    (3, "Star", 2, (1, 2, 1), (16, 2, 1), (31, 29, 27), "None", 0),
    (3, "Box", 1, (2, 1, 1), (8, 3, 1), (35, 26, 22), "Write", 16),
    (3, "Box", 2, (1, 1, 1), (16, 8, 1), (22, 21, 20), "None", 0),
    # tiles wider than a 256-element TMA box (cp.async loaders)
    (2, "Box", 6, (8, 1, 1), (32, 1, 1), (300, 30, 1), "None", 0),
    (3, "Star", 2, (2, 2, 1), (128, 1, 1), (290, 12, 10), "Read", 16),
]


@pytest.mark.parametrize("case", PIPE_CASES, ids=lambda c: "%dD_%s_r%d_c%s_b%s" % (c[0], c[1], c[2], c[3], c[4]))
@pytest.mark.parametrize("es", [8, 4])
def test_pipe_addressing_model(case, es):
    d, sh, r, c, blk, n, al, cl = case
    spec = O.make_spec(d, sh, "Row", "Jacobi", r, c[0], c[1], c[2], al, cl)
    g = O.geometry(spec, *n)
    for nctas in (0, 1, 3, 7):
        for chunk, depth in ((0, 0), (1, 1), (3, 2), (5, 1)):
            cnt = pipe_model.simulate(d, sh, r, c, blk, g.grid, g.left_offset, g.right_offset, al != "None",
                                      es=es, num_sms=2, occ=2, chunk=chunk, depth=depth, nctas=nctas)
            assert cnt is None or cnt > 0


@pytest.mark.parametrize("seed", range(6))
def test_batch_work_split_covers_every_plane_once(seed):
    """The batched kernel's split of the concatenated (grid, tile, plane) list over CTAs: every
    output plane of every tile of every grid is swept exactly once, by pieces that stay inside one
    tile of one grid (grids with no planes included)."""
    from pipe_model import batch_pieces

    rng = np.random.default_rng(seed)
    ng = int(rng.integers(1, 40))
    grids, first = [], 0
    for _ in range(ng):
        tiles = int(rng.integers(1, 9))
        m = int(rng.integers(0, 30)) if rng.random() < 0.2 else int(rng.integers(1, 30))
        grids.append((first, tiles, m))
        first += tiles * m
    total = first
    if total == 0:
        return
    for nctas in (1, 2, 7, 148, 296, total, total + 5):
        per = max(1, -(-total // nctas))
        seen = {}
        for b, gi, tile, zs, ze in batch_pieces(grids, total, per):
            f, tiles, m = grids[gi]
            assert m > 0 and 0 <= tile < tiles and 0 <= zs < ze <= m
            for z in range(zs, ze):
                key = (gi, tile, z)
                assert key not in seen
                seen[key] = b
        assert len(seen) == total


@pytest.mark.parametrize("dim", [2, 3])
def test_pair_cp_async_fill_equals_element_fill(dim):
    """The FP32 pair loader (two elements per cp.async, even pitch) fills every ring chunk exactly
    like the element loader: same global point (or zero fill) at every ring offset."""
    from pipe_model import copy_chunk

    rng = np.random.default_rng(dim)
    for _ in range(40):
        vec = 4
        pw = int(rng.integers(2, 20)) * vec
        rows = int(rng.integers(1, 12)) if dim == 3 else 1
        chp = int(rng.integers(1, 6))
        xdim = int(rng.integers(1, 60)) * 2
        ydim = int(rng.integers(3, 40))
        zdim = int(rng.integers(3, 30)) if dim == 3 else 1
        xl = int(rng.integers(0, max(1, xdim // vec + 2))) * vec
        y0 = int(rng.integers(0, ydim + 3))
        m0 = int(rng.integers(0, (zdim if dim == 3 else ydim) + 3))
        one = copy_chunk(dim, 1, pw, rows, chp, xl, y0, m0, xdim, ydim, zdim)
        two = copy_chunk(dim, 2, pw, rows, chp, xl, y0, m0, xdim, ydim, zdim)
        assert one == two


@pytest.mark.parametrize("R, left", [(1, 0), (3, 0), (6, 0), (8, 0), (2, 5)])
def test_tensor_core_operand_layouts_reproduce_the_stencil(R, left):
    """The tensor-core sweep's banded contraction, with operands laid out as tcs_tc.cu writes them
    and read as the tcgen05 K-major no-swizzle descriptors address them, equals the stencil on a
    tile (values exact in BF16, so hi = value and the contraction is exact in float64)."""
    from tc_model import TM, TN, tile_product

    rng = np.random.default_rng(R)
    D = 2 * R + 1
    mask2d = rng.integers(-4, 5, size=(D, D)).astype(np.float64)
    ydim, xdim = TM + 2 * R + 37, left + TN + 2 * R + 45
    grid = rng.integers(-8, 9, size=(ydim, xdim)).astype(np.float64)
    x0 = R + left
    for ty, tx in ((0, 0), (0, 1)):
        acc = tile_product(grid, mask2d, R, x0, ty, tx)
        for m in range(0, TM, 7):
            for n in range(TN):
                y, x = R + ty * TM + m, x0 + tx * TN + n
                if y + R >= ydim or x + R >= xdim:
                    continue
                want = sum(mask2d[dy + R, dx + R] * grid[y + dy, x + dx]
                           for dy in range(-R, R + 1) for dx in range(-R, R + 1))
                assert acc[m, n] == want, (m, n)


@pytest.mark.parametrize("es", [8, 4])
@pytest.mark.parametrize("shape", ["Box", "Star"])
@pytest.mark.parametrize("R", [1, 2, 3, 6, 8])
def test_temporal_blocking_model(R, shape, es):
    """tcs_tb2's tiles and phases (tests/tb_model.py): every shared-memory access stays inside its
    tile, the shared memory fits, every interior point is written once and nothing else, and one
    pass equals two plain sweeps (integer data and weights: exact in any order).  Grids: the
    smallest interior, ragged sizes, and Write-style left and right padding."""
    from tb_model import footprint, plain_sweep, sweep_tb2

    rng = np.random.default_rng(R * 10 + es)
    w = {o: int(rng.integers(-3, 4)) for o in footprint(shape, R)}
    for xdim, ydim, left, right in ((2 * R + 3, 2 * R + 2, 0, 0), (150, 45, 0, 0), (300, 81, 3, 5)):
        x0, x_lim, y_lim = R + left, xdim - R - right, ydim - R
        a = rng.integers(-9, 10, size=(ydim, xdim)).astype(np.int64)
        want = plain_sweep(plain_sweep(a, R, w, x0, x_lim, y_lim), R, w, x0, x_lim, y_lim)
        got, writes = sweep_tb2(a, shape, R, w, es, x0, x_lim, y_lim)
        interior = np.zeros(a.shape, dtype=bool)
        interior[R:y_lim, x0:x_lim] = True
        assert np.all(writes[interior] == 1) and np.all(writes[~interior] == 0)
        assert np.array_equal(got, want)


COMP_CASES = [
    ((2, "Box", "Row", "Variable", 6, 4, 1, 1, "None", 0), (301, 207, 1)),
    ((3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16), (60, 44, 38)),
    ((2, "Box", "Column", "Jacobi", 3, 2, 2, 1, "None", 0), (150, 99, 1)),
    ((3, "Box", "Row", "Variable", 2, 1, 2, 2, "Write", 8), (41, 37, 29)),
]


@pytest.mark.parametrize("case", COMP_CASES, ids=lambda c: ref_configs.key(c[0]))
def test_compensated_arithmetic_within_rounding_of_fp64(case):
    """The host build of the compensated FP32 arithmetic (tcs_tile.cuh with TCS_COMP): within
    3 * 2^-24 |exact| + 4 S 2^-48 sum |m||in| of the float64 oracle on the same FP32 inputs and
    FP32-rounded mask, the bound the GPU test applies to the f32c kernels; plain FP32 does worse
    on the long Variable stencils; border and padding untouched."""
    cfg, sides = case
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec = O.make_spec(*cfg)
    g = O.geometry(spec, *sides)
    shape = (g.grid[1], g.grid[0]) if d == 2 else (g.grid[2], g.grid[1], g.grid[0])
    rng = np.random.default_rng(r)
    a = rng.uniform(-1, 1, shape).astype(np.float32)
    S = O.stencil_size(spec)
    mask = rng.standard_normal(S) / S if c == "Variable" else None
    out_c = host_tile.sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, 1, mask, "f32c").astype(np.float64)
    out_p = host_tile.sweeps(cfg, a, g.grid, g.left_offset, g.right_offset, 1, mask, "f32").astype(np.float64)
    m32 = None if mask is None else mask.astype(np.float32).astype(np.float64)
    exact = O.sweep(spec, a.astype(np.float64), g.right_offset, m32)
    x0, x_lim = r + g.left_offset, g.grid[0] - r - (g.right_offset if al != "None" else 0)
    sl = (slice(r, g.grid[1] - r), slice(x0, x_lim)) if d == 2 else \
        (slice(r, g.grid[2] - r), slice(r, g.grid[1] - r), slice(x0, x_lim))
    mag = O.sweep(spec, np.abs(a.astype(np.float64)), g.right_offset, None if m32 is None else np.abs(m32))[sl]
    bound = 3 * 2.0 ** -24 * np.abs(exact[sl]) + 4 * S * 2.0 ** -48 * mag
    err_c, err_p = np.abs(out_c[sl] - exact[sl]), np.abs(out_p[sl] - exact[sl])
    assert np.all(err_c <= bound), float((err_c / bound).max())
    if c == "Variable" and r >= 4:
        assert err_c.max() < err_p.max()
    outside = np.ones(shape, dtype=bool)
    outside[sl] = False
    assert np.array_equal(out_c[outside], a.astype(np.float64)[outside])
