"""Parameter sets for which the reference's own kernels are generated and built (test infrastructure).

Each entry is one generated ``kernels.cu``: (dimension, neighbourhood, orientation, coefficients,
range, cx, cy, cz, alignment, cl_size).  The list spans every generator switch — 2D/3D, Box/Star,
Row/Column, Jacobi/Variable, None/Read/Write, odd and even ranges and coarsening factors — plus
the parameter sets of the benchmark workloads.
"""

from __future__ import annotations

PARITY = [
    # 2D, every switch at small sizes
    (2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0),
    (2, "Box", "Column", "Jacobi", 2, 2, 3, 1, "None", 0),
    (2, "Box", "Row", "Variable", 2, 3, 2, 1, "Read", 16),
    (2, "Box", "Column", "Variable", 1, 2, 2, 1, "Write", 16),
    (2, "Star", "Row", "Jacobi", 3, 2, 1, 1, "Write", 8),
    (2, "Star", "Column", "Jacobi", 1, 1, 4, 1, "None", 0),
    (2, "Star", "Row", "Variable", 4, 4, 2, 1, "Read", 16),
    (2, "Star", "Column", "Variable", 2, 3, 3, 1, "Write", 16),
    (2, "Box", "Row", "Variable", 6, 2, 2, 1, "None", 0),
    # 3D, every switch
    (3, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0),
    (3, "Box", "Column", "Jacobi", 1, 2, 2, 2, "Read", 16),
    (3, "Box", "Row", "Variable", 2, 2, 1, 2, "Write", 16),
    (3, "Box", "Column", "Variable", 1, 1, 3, 1, "None", 0),
    (3, "Star", "Row", "Jacobi", 2, 2, 2, 2, "None", 0),
    (3, "Star", "Column", "Jacobi", 3, 1, 2, 3, "Write", 8),
    (3, "Star", "Row", "Variable", 4, 1, 1, 1, "Read", 16),
    (3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16),
    (3, "Star", "Column", "Variable", 2, 3, 1, 2, "Read", 16),
]

# Further parameter sets that pin the CPU oracle only (fixtures from the reference's generated
# kernels through the host shim; no GPU test runs them): the long ranges 5-8, 3D Box beyond range 1,
# 3D Star Column at range 4, and coarsening factors of 4 in 3D.
EXTRA = [
    (2, "Box", "Row", "Jacobi", 5, 1, 2, 1, "Read", 8),
    (2, "Box", "Column", "Variable", 7, 2, 1, 1, "None", 0),
    (2, "Star", "Row", "Variable", 8, 2, 4, 1, "Write", 16),
    (2, "Star", "Column", "Jacobi", 6, 4, 1, 1, "Read", 16),
    (3, "Box", "Row", "Variable", 3, 1, 2, 1, "Read", 8),
    (3, "Box", "Column", "Jacobi", 2, 2, 1, 2, "None", 0),
    (3, "Star", "Column", "Variable", 4, 1, 2, 2, "Write", 16),
    (3, "Star", "Row", "Jacobi", 5, 4, 1, 1, "None", 0),
]

# Parameter sets timed on the GPU for the benchmark workloads.
BENCH = [
    (2, "Box", "Row", "Jacobi", 1, 1, 1, 1, "None", 0),
    (2, "Box", "Row", "Jacobi", 1, 1, 2, 1, "None", 0),
    (2, "Box", "Row", "Jacobi", 1, 2, 2, 1, "None", 0),
    (3, "Star", "Row", "Variable", 4, 1, 1, 1, "Read", 16),
    (3, "Star", "Row", "Variable", 4, 1, 1, 2, "Read", 16),
    (3, "Star", "Row", "Variable", 4, 2, 2, 1, "Read", 16),
    (3, "Star", "Row", "Variable", 4, 1, 2, 2, "Read", 16),
    (3, "Star", "Row", "Variable", 4, 2, 2, 2, "Read", 16),
    (3, "Star", "Row", "Variable", 4, 4, 2, 1, "Read", 16),
    (3, "Star", "Row", "Variable", 4, 1, 4, 2, "Read", 16),
    (3, "Star", "Row", "Variable", 4, 3, 4, 3, "Read", 16),  # best of the launch-shape sweep (ref_sweep.py)
    (2, "Box", "Row", "Variable", 6, 1, 1, 1, "None", 0),
    (2, "Box", "Row", "Variable", 6, 2, 2, 1, "None", 0),
    (2, "Box", "Row", "Variable", 6, 4, 4, 1, "None", 0),
    (2, "Box", "Row", "Variable", 6, 2, 4, 1, "None", 0),
]


def key(cfg) -> str:
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    k = "%dD_%s_%s_%s_r%d_c%dx%d" % (d, sh, o, c, r, cx, cy)
    if d == 3:
        k += "x%d" % cz
    k += "_%s%d" % (al, cl)
    return k


ALL = list(dict.fromkeys(PARITY + BENCH))
