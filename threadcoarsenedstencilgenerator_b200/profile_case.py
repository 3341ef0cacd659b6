"""Run a few sweeps of a benchmark workload on a reduced grid, for profilers.

    python -m threadcoarsenedstencilgenerator_b200.profile_case --workload 3d_star_var_r4_512 \
        --grid 256 256 256 --sweeps 3

    python -m threadcoarsenedstencilgenerator_b200.profile_case --workload batch_3d_star_jacobi_r2_64 \
        --grids 16 --sweeps 3 --precision f32
    python -m threadcoarsenedstencilgenerator_b200.profile_case --workload 2d_box_var_r6_16384x8192 \
        --grid 16384 8192 --sweeps 3 --precision f32 --tensor-cores
    python -m threadcoarsenedstencilgenerator_b200.profile_case --workload 2d_box_jacobi_r1_4096 \
        --grid 4096 4096 --sweeps 4 --temporal

The workload's tuned launch (tuned.json) and seeded data are used.  Keep the grid above the L2
size (126 MB per buffer) so that DRAM counters stay meaningful, and small enough for an ncu
capture to finish in a minute or two.  For a batch workload, `--grids K` keeps its first K grids
and each sweep is one batched launch.
"""

from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200.workloads import BATCH_WORKLOADS, WORKLOADS

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", required=True, choices=sorted(WORKLOADS) + sorted(BATCH_WORKLOADS))
    ap.add_argument("--grid", type=int, nargs="+")
    ap.add_argument("--grids", type=int, default=0, help="batch workloads: first K grids (0 = all)")
    ap.add_argument("--sweeps", type=int, default=3)
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"])
    ap.add_argument("--tensor-cores", action="store_true", help="2D Box FP32: the tcgen05 sweep")
    ap.add_argument("--temporal", action="store_true", help="2D: two sweeps per pass (tcs_tb2)")
    a = ap.parse_args(argv)
    if a.workload in BATCH_WORKLOADS:
        return _batch(a)
    if not a.grid:
        ap.error("--grid is required for single-grid workloads")
    w = WORKLOADS[a.workload]
    spec = w.tuned_spec().replace(precision=a.precision)
    launch = w.tuned_launch()
    grid = tuple(a.grid) + (1,) * (3 - len(a.grid))
    geom = spec.geometry(*grid)
    st = tcs.Stencil(spec)
    m = w.make_mask()
    if m is not None:
        st.copy_mask(m)
    dt = torch.float64 if a.precision == "f64" else torch.float32
    x = torch.from_numpy(w.make_input(geom)).to("cuda", dtype=dt)
    y = x.clone()
    if a.temporal:
        st.sweeps_tb2(geom, x, y, a.sweeps)
    for _ in range(0 if a.temporal else a.sweeps):
        if a.tensor_cores:
            st.tc_update_grid(geom, x, y)
        else:
            st.update_grid(geom, x, y, launch)
        x, y = y, x
    torch.cuda.synchronize()
    if st.device_status() != 0:
        print("device status word set", file=sys.stderr)
        return 1
    print("ok", a.workload, grid, st.plan(geom, launch))
    return 0


def _batch(a) -> int:
    import numpy as np
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200.batch import BatchedSweeps
    from threadcoarsenedstencilgenerator_b200.workloads import BATCH_WORKLOADS

    w = BATCH_WORKLOADS[a.workload]
    spec = w.spec.replace(precision=a.precision)
    geoms = w.geometries(spec)
    arrs = w.make_inputs(geoms, np.float64 if a.precision == "f64" else np.float32)
    if a.grids:
        geoms, arrs = geoms[:a.grids], arrs[:a.grids]
    st = tcs.Stencil(spec)
    xs = [torch.from_numpy(v).cuda() for v in arrs]
    ys = [x.clone() for x in xs]
    bt = BatchedSweeps(st, geoms, xs, ys, w.tuned_launch(a.precision))
    bt.sweeps(a.sweeps)
    torch.cuda.synchronize()
    if st.device_status() != 0:
        print("device status word set", file=sys.stderr)
        return 1
    print("ok", a.workload, len(geoms), "grids", sum(g.interior_points for g in geoms), "points", bt.plan())
    bt.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
