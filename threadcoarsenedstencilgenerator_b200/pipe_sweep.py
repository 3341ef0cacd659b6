"""Exhaustive timing of pipelined-sweep launch shapes on a benchmark workload.

    python -m threadcoarsenedstencilgenerator_b200.pipe_sweep --workload 3d_star_var_r4_512

The reference picks a block shape by timing every candidate (Benchmark2D / Benchmark3D,
cuda/benchmark.cpp:223-320); this does the same for the engine's pipe kernel, whose shape also has
a thread coarsening and the planes per ring chunk.  Each shape runs the workload's grid and seeded data for --warmup then --sweeps sweeps
timed with CUDA events; one JSON line per shape (GLup/s, or the planner's reason for rejecting it),
then the best shapes.  Shapes the planner rejects (shared memory, TMA box limits) are skipped.
"""

from __future__ import annotations

import argparse
import json
import sys


def _pairs(vals):
    return [tuple(int(v) for v in s.split("x")) for s in vals]


def main(argv=None) -> int:
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="3d_star_var_r4_512", choices=sorted(WORKLOADS))
    ap.add_argument("--coarsening", nargs="+", default=["1x2", "1x4", "2x2", "2x4", "4x2", "1x8"],
                    help="cx x cy thread coarsenings (cz = 1)")
    ap.add_argument("--blocks", nargs="+", default=["32x4", "32x8", "64x2", "64x4", "128x2"])
    ap.add_argument("--chunks", type=int, nargs="+", default=[2, 3])
    ap.add_argument("--sweeps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"])
    a = ap.parse_args(argv)
    w = WORKLOADS[a.workload]
    base = w.tuned_spec().replace(precision=a.precision)
    geom = base.geometry(*w.grid)
    dt = torch.float64 if base.precision == "f64" else torch.float32
    x = torch.from_numpy(w.make_input(geom)).to("cuda", dtype=dt)
    y = x.clone()
    mask = w.make_mask()
    stream = torch.cuda.current_stream()
    results = []
    for cx, cy in _pairs(a.coarsening):
        st = tcs.Stencil(base.replace(cx=cx, cy=cy, cz=1))
        if mask is not None:
            st.copy_mask(mask)
        for bx, by in _pairs(a.blocks):
            for ch in a.chunks:
                launch = tcs.Launch(block=(bx, by, 1), variant="pipe", chunk=ch)
                rec = {"coarsening": [cx, cy, 1], "block": [bx, by, 1], "chunk": ch}
                try:
                    plan = st.plan(geom, launch)
                except tcs.TcsError as e:
                    rec["rejected"] = str(e)
                    print(json.dumps(rec), flush=True)
                    continue
                st.sweeps(geom, x, y, a.warmup, launch, stream)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                st.sweeps(geom, x, y, a.sweeps, launch, stream)
                e1.record(stream)
                torch.cuda.synchronize()
                if st.device_status() != 0:
                    print("device status word set", file=sys.stderr)
                    return 1
                rec.update(glups=geom.interior_points * a.sweeps / (e0.elapsed_time(e1) / 1e3) / 1e9,
                           ctas_per_sm=plan.ctas_per_sm, depth=plan.depth)
                results.append(rec)
                print(json.dumps(rec), flush=True)
    results.sort(key=lambda r: -r["glups"])
    print(json.dumps({"best": results[:5]}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
