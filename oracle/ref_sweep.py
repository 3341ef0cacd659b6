"""Launch-shape sweep of the reference's own generated kernel on the 3D Star Variable r4 workload.

The reference chooses its launch by timing every thread-block shape (Benchmark3D,
cuda/benchmark.cpp:287-318, shapes from cuda/primes.cpp:74-87) for one generated kernel, i.e. for
one coarsening triple baked in by the generator.  The workload's specification asks for the best
over coarsening factors 1..4 per axis and all block shapes.  This recipe

  build  generates and compiles the reference's kernel for all 64 coarsening triples (1..4 per
         axis) of 3D Star Row Variable range 4 with Read alignment to 16 points, with the recipe
         of build_ref.py (outputs into oracle/_ref/, never committed);
  run    times each triple on the 512^3 grid (CUDA events around back-to-back launches after
         warm-up launches, ref_time in ref_driver.cu) over a stated subset of the reference's
         block enumeration: the 3D shapes of primes.cpp with 128, 256 or 512 threads and an x
         extent of at least 16 (narrower x blocks break the coalescing of the row-major rows the
         kernel reads), writing one JSON line per (triple, block) and the best shape per triple.

This measures the reference, to choose the reference shape that bench.py times beside the
engine.  It loads only oracle/_ref libraries and the block enumeration's plain-Python file.

    TCS_REFERENCE_ROOT=<reference tree> python oracle/ref_sweep.py build
    python oracle/ref_sweep.py run --out gpurun_out/ref_sweep.jsonl
"""

from __future__ import annotations

import argparse
import ctypes
import itertools
import json
import sys
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

from oracle.ref_configs import key  # noqa: E402

GRID = (512, 512, 512)
R = 4
TRIPLES = list(itertools.product(range(1, 5), repeat=3))


def cfg_of(c):
    return (3, "Star", "Row", "Variable", R, c[0], c[1], c[2], "Read", 16)


def lib_path(c) -> Path:
    return HERE / "_ref" / key(cfg_of(c)) / "libref.so"


def block_subset() -> list:
    """3D shapes of the reference's enumeration (cuda/primes.cpp order, as restated by the engine's
    primes.py, loaded from its file without importing the engine) with 128, 256 or 512 threads and
    x extent >= 16."""
    import importlib.util

    path = HERE.parent / "threadcoarsenedstencilgenerator_b200" / "primes.py"
    spec = importlib.util.spec_from_file_location("tcs_primes", path)
    primes = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(primes)
    return [tuple(b) for b in primes.block_shapes(3, 1024)
            if b[0] * b[1] * b[2] in (128, 256, 512) and b[0] >= 16]


def build(jobs: int = 8) -> list:
    from oracle.build_ref import compile_one, reference_available

    if not reference_available():
        raise SystemExit("reference tree not found; nothing built")
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        return list(ex.map(lambda c: compile_one(cfg_of(c)), TRIPLES))


def geometry(c):
    import oracle as O

    return O.geometry(O.make_spec(*cfg_of(c)), *GRID)


def time_shape(lib, g, block, warmup: int, sweeps: int) -> float | None:
    """GLup/s of one launch shape, or None when the shape does not launch (too many registers
    for the block, say)."""
    u3 = ctypes.c_uint * 3
    gb = tuple(max(1, -(-g.threads[i] // block[i])) for i in range(3))
    ms = ctypes.c_float()
    mask = (ctypes.c_double * 25)(*([1.0 / 25] * 25))
    rc = lib.ref_time(ctypes.c_uint(3), u3(*g.grid), u3(*block), u3(*gb), ctypes.c_uint(g.right_offset), mask,
                      ctypes.c_uint(25), ctypes.c_uint(warmup), ctypes.c_uint(sweeps), ctypes.byref(ms))
    if rc != 0 or ms.value <= 0:
        return None
    e = g.elements
    return e[0] * e[1] * e[2] * sweeps / (ms.value / 1e3) / 1e9


def run(out_path: Path | None, warmup: int, sweeps: int, triples=None) -> dict:
    blocks = block_subset()
    best = {}
    out = open(out_path, "a") if out_path else None
    t0 = time.perf_counter()
    for c in triples or TRIPLES:
        p = lib_path(c)
        if not p.exists():
            continue
        lib = ctypes.CDLL(str(p))
        g = geometry(c)
        for b in blocks:
            glups = time_shape(lib, g, b, warmup, sweeps)
            if out:
                out.write(json.dumps({"coarsening": list(c), "block": list(b), "glups": glups}) + "\n")
                out.flush()
            if glups is not None and glups > best.get(c, (0.0, None))[0]:
                best[c] = (glups, b)
        if c in best:
            print(json.dumps({"coarsening": list(c), "best_glups": round(best[c][0], 2),
                              "best_block": list(best[c][1])}), flush=True)
    ranked = sorted(best.items(), key=lambda kv: -kv[1][0])
    summary = {"triples": len(best), "blocks_per_triple": len(blocks), "seconds": time.perf_counter() - t0,
               "top": [{"coarsening": list(c), "glups": round(v[0], 2), "block": list(v[1])} for c, v in ranked[:10]]}
    print(json.dumps(summary))
    return summary


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["build", "run"])
    ap.add_argument("--out", type=Path)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--sweeps", type=int, default=5)
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    if a.cmd == "build":
        print("built %d reference kernels" % len(build(a.j)))
        return 0
    run(a.out, a.warmup, a.sweeps)
    return 0


if __name__ == "__main__":
    sys.exit(main())
