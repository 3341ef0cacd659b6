"""Run a few sweeps of a benchmark workload on a reduced grid, for profilers.

    python -m threadcoarsenedstencilgenerator_b200.profile_case --workload 3d_star_var_r4_512 \
        --grid 256 256 256 --sweeps 3

The workload's tuned launch (tuned.json) and seeded data are used.  Keep the grid above the L2
size (126 MB per buffer) so that DRAM counters stay meaningful, and small enough for an ncu
capture to finish in a minute or two.
"""

from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", required=True, choices=sorted(WORKLOADS))
    ap.add_argument("--grid", type=int, nargs="+", required=True)
    ap.add_argument("--sweeps", type=int, default=3)
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"])
    a = ap.parse_args(argv)
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
    for _ in range(a.sweeps):
        st.update_grid(geom, x, y, launch)
        x, y = y, x
    torch.cuda.synchronize()
    if st.device_status() != 0:
        print("device status word set", file=sys.stderr)
        return 1
    print("ok", a.workload, grid, st.plan(geom, launch))
    return 0


if __name__ == "__main__":
    sys.exit(main())
