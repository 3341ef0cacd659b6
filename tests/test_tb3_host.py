"""The two-sweep kernel's control flow (3D, and 2D strips) on the CPU (tests/host_tile/tb3_host.cpp): one pass
equals two oracle sweeps bit for bit -- extended and output tiles, ragged last tiles, the border
copy into the plane buffer, pieces that restart both pipelines, the slot rotation at chunk ends."""

import numpy as np
import pytest

import host_tile
import oracle as O

CASES = [
    # (cfg, grid, block (threads), piece, unroll)
    ((3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0), (37, 29, 23), (8, 6), 7, 2),
    ((3, "Star", "Row", "Variable", 2, 1, 1, 1, "Read", 16), (45, 26, 19), (16, 4), 1 << 30, 3),
    ((3, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0), (29, 23, 17), (8, 8), 5, 2),
    ((3, "Box", "Column", "Variable", 1, 2, 1, 1, "Write", 8), (33, 20, 15), (6, 5), 4, 1),
    ((3, "Star", "Column", "Variable", 3, 1, 1, 1, "Write", 8), (41, 30, 22), (12, 10), 6, 2),
    ((3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16), (52, 40, 26), (10, 8), 9, 3),
    ((3, "Box", "Row", "Variable", 2, 2, 2, 1, "None", 0), (31, 27, 16), (6, 6), 1 << 30, 2),
    # 2D: strips marching along y (block[1] ignored)
    ((2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0), (45, 37, 1), (10, 1), 9, 8),
    ((2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0), (33, 30, 1), (8, 1), 1 << 30, 3),
    ((2, "Star", "Row", "Variable", 2, 2, 1, 1, "Read", 8), (52, 41, 1), (8, 1), 11, 5),
    ((2, "Box", "Row", "Variable", 3, 1, 1, 1, "Write", 8), (47, 35, 1), (12, 1), 7, 7),
    ((2, "Star", "Row", "Jacobi", 4, 2, 1, 1, "None", 0), (61, 44, 1), (10, 1), 1 << 30, 8),
]


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "%s_%s_%s_r%d_b%dx%d" % (c[0][1], c[0][2], c[0][3], c[0][4],
                                                                             c[2][0], c[2][1]))
def test_two_sweep_pass_equals_two_sweeps(case, precision):
    cfg, n, block, piece, unroll = case
    spec = O.make_spec(*cfg)
    g = O.geometry(spec, *n)
    rng = np.random.default_rng(61)
    dt = np.float64 if precision == "f64" else np.float32
    shape = (g.grid[2], g.grid[1], g.grid[0]) if cfg[0] == 3 else (g.grid[1], g.grid[0])
    a = rng.uniform(-1, 1, shape).astype(dt)
    mask = rng.standard_normal(O.stencil_size(spec)) if cfg[3] == "Variable" else None
    want = O.sweeps(spec, a, 4, g.right_offset, mask)
    got = host_tile.tb3_passes(cfg, a, g.grid, g.left_offset, g.right_offset, 2, mask, precision, block, piece,
                               unroll)
    assert np.array_equal(got, want)


def test_2d_strip_instances_compile_and_reject_what_they_cannot_run():
    """The 2D two-sweep kernel instantiates without a GPU for Row stencils of several ranges (its
    default strip of 64 threads, narrowed where a TMA box needs it) and rejects Column order and
    FP32 with an odd range (no output strip of 16-byte multiples)."""
    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200.stencil import precompile_tb3

    for sh, co, r, prec in [("Box", "Jacobi", 1, "f64"), ("Star", "Variable", 3, "f64"),
                            ("Box", "Variable", 6, "f64"), ("Star", "Jacobi", 2, "f32")]:
        spec = tcs.StencilSpec(dimension=2, neighbourhood=sh, coefficients=co, range=r, precision=prec)
        assert precompile_tb3(spec).endswith(".cubin")
    with pytest.raises(tcs.UnsupportedLaunch):
        precompile_tb3(tcs.StencilSpec(dimension=2, neighbourhood="Star", orientation="Column", range=1))
    with pytest.raises(tcs.UnsupportedLaunch):
        precompile_tb3(tcs.StencilSpec(dimension=2, neighbourhood="Box", range=1, precision="f32"))


@pytest.mark.parametrize("R", range(1, 9))
def test_2d_strip_row_buffer_fits_the_host_allocation(R):
    """The 2D strip kernel's row buffer (left margin TB_ML = R rounded up to even, width rounded up
    to even: tcs_kernels.cuh) never exceeds the EX + 2R + 2 elements per buffer that the host
    reserves (tcs_capi.cpp, resolve_tb3), and every thread's column pair starts on an even column."""
    for EX in range(2 * R + 2, 258, 2):
        ml = R + (R & 1)
        bw = ((ml + EX + R + 1) // 2) * 2
        assert bw <= EX + 2 * R + 2 and bw % 2 == 0 and ml % 2 == 0
        assert all((ml + ex0) % 2 == 0 for ex0 in range(0, EX, 2))
        # stage 2 reads columns ml + ex0 - R .. ml + ex0 + 1 + R of the buffer: inside it
        assert ml - R >= 0 and ml + (EX - 2) + 1 + R < bw
