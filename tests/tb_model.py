"""CPU model of the tcs_tb2 kernel (two sweeps per pass over HBM, 2D), used by
tests/test_kernel_host.py.

Transcribes the launch of ``launch_tb2`` (tcs_capi.cpp: output tile 128 x 256/es, thread tile
1 x 8, one CTA per output tile over the interior, the dynamic shared-memory size) and the indexing
of ``tcs_tb2`` (tcs_kernels.cuh): the input tile's copies (zero outside the grid), the first-sweep
tile written from thread tiles with its interior select, and the second sweep into the output.
Every shared-memory index the thread tiles read or write is checked against the tile it addresses,
and every stage-2 read must hit a value stage 1 wrote.  The tiles carry values, so the model also
checks the result: on integer data with integer weights (exact sums in any order) one pass equals
two plain sweeps, with every interior point written once and no other point written.
"""

from __future__ import annotations

import numpy as np

from march_model import cdiv

TB_TX, TB_CX, TB_CY, TB_THREADS = 128, 1, 8, 256
SMEM_OPTIN = 232448  # bytes of dynamic shared memory a B200 CTA may opt in to


def tb_ty(es: int) -> int:
    return 256 // es


def tiles(R: int, es: int):
    """(BW, BH, AW, AH): first-sweep tile rounded to thread tiles, and the input tile."""
    bw = cdiv(TB_TX + 2 * R, TB_CX) * TB_CX
    bh = cdiv(tb_ty(es) + 2 * R, TB_CY) * TB_CY
    return bw, bh, bw + 2 * R, bh + 2 * R


def smem_bytes(R: int, es: int) -> int:
    """launch_tb2's dynamic shared memory: ((bw + 2R)(bh + 2R) + bw bh) elements."""
    bw = cdiv(TB_TX + 2 * R, TB_CX) * TB_CX
    bh = cdiv(tb_ty(es) + 2 * R, TB_CY) * TB_CY
    return ((bw + 2 * R) * (bh + 2 * R) + bw * bh) * es


def footprint(shape: str, R: int):
    """(dx, dy) offsets of one output's terms (the order does not matter for exact sums)."""
    if shape == "Box":
        return [(dx, dy) for dy in range(-R, R + 1) for dx in range(-R, R + 1)]
    return sorted({(dx, 0) for dx in range(-R, R + 1)} | {(0, dy) for dy in range(-R, R + 1)})


def plain_sweep(a: np.ndarray, R: int, w: dict, x0: int, x_lim: int, y_lim: int) -> np.ndarray:
    """One sweep of the interior [x0, x_lim) x [R, y_lim); every other point keeps its value."""
    out = a.copy()
    acc = np.zeros((y_lim - R, x_lim - x0), dtype=np.int64)
    for (dx, dy), m in w.items():
        acc += m * a[R + dy:y_lim + dy, x0 + dx:x_lim + dx]
    out[R:y_lim, x0:x_lim] = acc
    return out


def _stage(src, sw, tiles_w, tiles_h, off, fp, w, size_src):
    """Thread tiles (r0, c0) over a tiles_w x tiles_h grid of 1 x 8 tiles reading `src` (flat,
    row width sw) at row/column offset `off`: returns (r0, c0, base index, [sum for each of the 8
    outputs]) after checking every index the traversal loads."""
    t = np.arange(tiles_w * tiles_h)
    r0 = (t // tiles_w) * TB_CY
    c0 = (t % tiles_w) * TB_CX
    base = (r0 + off) * sw + (c0 + off)
    vals = []
    for ey in range(TB_CY):
        acc = np.zeros(len(t), dtype=np.int64)
        for (dx, dy) in fp:
            idx = base + dx + (ey + dy) * sw
            assert idx.min() >= 0 and idx.max() < size_src, "shared-memory read outside its tile"
            v = src[idx]
            assert not np.any(v == np.iinfo(np.int64).min), "read a shared value no stage wrote"
            acc += w[(dx, dy)] * v
        vals.append(acc)
    return r0, c0, base, vals


def sweep_tb2(a: np.ndarray, shape: str, R: int, w: dict, es: int, x0: int, x_lim: int, y_lim: int):
    """One tcs_tb2 launch over grid `a` (int64, rows y, columns x): returns (out, writes).  `out`
    starts as a copy of `a`, as the second ping-pong buffer carries the same border."""
    ydim, xdim = a.shape
    ty = tb_ty(es)
    BW, BH, AW, AH = tiles(R, es)
    assert smem_bytes(R, es) == (AW * AH + BW * BH) * es <= SMEM_OPTIN
    assert TB_TX % TB_CX == 0 and ty % TB_CY == 0
    fp = footprint(shape, R)
    hole = np.iinfo(np.int64).min
    out = a.copy()
    writes = np.zeros(a.shape, dtype=np.int64)
    ex, ey = max(0, x_lim - x0), y_lim - R
    gx_n, gy_n = max(1, cdiv(ex, TB_TX)), max(1, cdiv(ey, ty))
    for by in range(gy_n):
        for bx in range(gx_n):
            xs, ys = x0 + bx * TB_TX, R + by * ty
            # input tile: q -> (r, cc), zero outside the grid
            q = np.arange(AW * AH)
            r, cc = q // AW, q % AW
            gy, gx = ys - 2 * R + r, xs - 2 * R + cc
            inside = (gy >= 0) & (gy < ydim) & (gx >= 0) & (gx < xdim)
            A = np.where(inside, a[np.clip(gy, 0, ydim - 1), np.clip(gx, 0, xdim - 1)], 0).astype(np.int64)
            # stage 1: first sweep on the (BH x BW) tile; points outside the interior keep their value
            Bt = np.full(BW * BH, hole, dtype=np.int64)
            r0, c0, base, vals = _stage(A, AW, BW // TB_CX, BH // TB_CY, R, fp, w, AW * AH)
            for e in range(TB_CY):
                gy1, gx1 = ys - R + r0 + e, xs - R + c0
                interior = (gx1 >= x0) & (gx1 < x_lim) & (gy1 >= R) & (gy1 < y_lim)
                bi = (r0 + e) * BW + c0
                assert bi.min() >= 0 and bi.max() < BW * BH
                Bt[bi] = np.where(interior, vals[e], A[base + e * AW])
            # stage 2: second sweep of the (ty x 128) output tile
            r0, c0, _, vals = _stage(Bt, BW, TB_TX // TB_CX, ty // TB_CY, R, fp, w, BW * BH)
            for e in range(TB_CY):
                gy2, gx2 = ys + r0 + e, xs + c0
                ok = (gx2 < x_lim) & (gy2 < y_lim)
                out[gy2[ok], gx2[ok]] = vals[e][ok]
                np.add.at(writes, (gy2[ok], gx2[ok]), 1)
    return out, writes
