"""CPU model of the tensor-core sweep (tcs_tc.cu): the operand layouts the kernel writes and the
tcgen05 canonical K-major no-swizzle layout the tensor core reads, and the banded contraction.

Element (row i, column k) of an operand with start address s, leading byte offset LBO (between
the two 16-byte K halves) and stride byte offset SBO (between 8-row core-matrix groups) lives at
s + (i % 8) * 16 + (i // 8) * SBO + (k % 8) * 2 + (k // 8) * LBO; one MMA reads rows 0..M-1 and
k = 0..15.  Used by tests/test_kernel_host.py.
"""

from __future__ import annotations

import numpy as np

TM, TN, KD, NCH = 128, 32, 48, 6


def read_operand(mem: dict, start: int, lbo: int, sbo: int, rows: int) -> np.ndarray:
    out = np.zeros((rows, 16))
    for i in range(rows):
        for k in range(16):
            out[i, k] = mem.get(start + (i % 8) * 16 + (i // 8) * sbo + (k % 8) * 2 + (k // 8) * lbo, 0.0)
    return out


BCOL = 2 * TN * 16   # bytes per 16-byte column of a row offset: high-part rows 0-31, low-part rows 32-63
BDY = NCH * BCOL


def b_operand(mask2d: np.ndarray, R: int) -> dict:
    """Toeplitz operands as built by tc_build (tcs_capi.cpp) (byte address -> value); the values are
    exact in BF16 here, so the high part is the value and the low part is zero."""
    D = 2 * R + 1
    mem = {}
    for dy in range(D):
        for ch in range(NCH):
            for n in range(TN):
                for e in range(8):
                    k = 8 * ch + e
                    j = k - n
                    if 0 <= j <= 2 * R:
                        mem[dy * BDY + ch * BCOL + n * 16 + e * 2] = mask2d[dy, j]
                        mem[dy * BDY + ch * BCOL + (TN + n) * 16 + e * 2] = 0.0
    return mem


def a_operand(grid: np.ndarray, R: int, x0: int, ty: int, tx: int) -> tuple:
    """Operand tile as written by load_split: (byte address -> value, column stride cs)."""
    rows = TM + 2 * R
    cs = ((rows * 16 + 127) // 128) * 128 + 16 if rows <= 142 else rows * 16  # col_stride in tcs_tc.cu
    ydim, xdim = grid.shape
    gy0 = ty * TM
    gx0 = x0 + tx * TN - R
    mem = {}
    for r in range(rows):
        for k in range(KD):
            gy, gx = gy0 + r, gx0 + k
            v = grid[gy, gx] if (k < TN + 2 * R and gy < ydim and gx < xdim) else 0.0
            mem[(k // 8) * cs + r * 16 + (k % 8) * 2] = v
    return mem, cs


def tile_product(grid: np.ndarray, mask2d: np.ndarray, R: int, x0: int, ty: int, tx: int) -> np.ndarray:
    """The accumulator of one tile: the sum over row offsets dy and K steps s of A_dy,s . B_dy,s^T,
    each operand read through its descriptor exactly as the kernel's issue loop encodes it."""
    amem, cs = a_operand(grid, R, x0, ty, tx)
    bmem = b_operand(mask2d, R)
    acc = np.zeros((TM, TN))
    for dy in range(2 * R + 1):
        for s in range(KD // 16):
            A = read_operand(amem, 2 * s * cs + dy * 16, cs, 128, TM)
            B = read_operand(bmem, dy * BDY + 2 * s * BCOL, BCOL, 128, 2 * TN)  # the N = 64 MMA
            P = A @ B.T
            acc += P[:, :TN] + P[:, TN:]  # hi*hi + hi*lo
    return acc
