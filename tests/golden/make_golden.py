"""Generate the golden fixtures of tests/golden/ from the reference's own generated kernels.

For every parameter set of ``oracle.ref_configs.PARITY`` (seeds 1000 + i; with ``--extra`` the
CPU-only sets of ``ref_configs.EXTRA``, seeds 2000 + i) this script
  1. runs the reference generators (through ``oracle.build_ref.generate``, i.e. straight from the
     read-only reference tree) to obtain that set's ``kernels.cu``;
  2. compiles it for the host CPU with ``ref_host_shim.cpp`` (g++ -O2 -mfma -ffp-contract=fast,
     the contraction nvcc applies by default);
  3. runs NSWEEPS ping-pong sweeps on a seeded grid (numpy default_rng(seed): interior and border
     U[0,1); Variable masks N(0,1) normalised to sum 1) and stores the result.

Each fixture ``<key>.npz`` holds the final grid plus everything needed to regenerate the input
(spec, raw grid size, seed, sweeps, mask), so the tests can check the oracle against it on any
machine.  ``--gpu`` instead takes the outputs from the reference kernels compiled for sm_100a
(``oracle/_ref/<key>/libref.so``, run on a B200) and writes them to ``--out``.

Run: ``python tests/golden/make_golden.py`` (needs the reference tree, g++).
"""

from __future__ import annotations

import argparse
import ctypes
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import ref_configs  # noqa: E402

NSWEEPS = 3
SIZES_2D = (37, 29)
SIZES_3D = (23, 19, 15)


def fixture_input(cfg, seed):
    """Seeded raw grid of the fixture (before the engine's padding): returns geometry + arrays."""
    import oracle as O

    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec = O.make_spec(d, sh, o, c, r, cx, cy, cz, al, cl)
    nx, ny, nz = (SIZES_2D + (1,)) if d == 2 else SIZES_3D
    g = O.geometry(spec, nx, ny, nz)
    rng = np.random.default_rng(seed)
    shape = (g.grid[1], g.grid[0]) if d == 2 else (g.grid[2], g.grid[1], g.grid[0])
    a = rng.random(shape)
    S = O.stencil_size(spec)
    mask = None
    if c == "Variable":
        m = rng.standard_normal(S)
        mask = m / m.sum()
    return spec, (nx, ny, nz), g, a, mask


def shim_outputs(cfg, seed, workdir: Path):
    from oracle.build_ref import generate

    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec, raw, g, a, mask = fixture_input(cfg, seed)
    dest = workdir / ref_configs.key(cfg)
    generate(cfg, dest)
    so = dest / "shim.so"
    cmd = ["g++", "-O2", "-mfma", "-ffp-contract=fast", "-shared", "-fPIC", "-DSHIM_DIM=%d" % d,
           "-DSHIM_ALIGNED=%d" % (0 if al == "None" else 1)] + (["-DSHIM_VARIABLE"] if c == "Variable" else []) + [
        "-I", str(dest), str(HERE / "ref_host_shim.cpp"), "-o", str(so)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(proc.stderr)
    lib = ctypes.CDLL(str(so))
    u3 = ctypes.c_uint * 3
    cz_ = cz if d == 3 else 1
    block = (8, 4, 2) if d == 3 else (8, 4, 1)
    thr = g.threads
    gb = tuple(-(-thr[i] // block[i]) for i in range(3))
    x = a.copy()
    y = a.copy()
    m = np.zeros(1) if mask is None else np.ascontiguousarray(mask)
    lib.shim_sweeps(u3(*g.grid), u3(*block), u3(*gb), ctypes.c_uint(g.right_offset),
                    m.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(m.size), x.ctypes.data_as(ctypes.c_void_p),
                    y.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(NSWEEPS))
    out = y if NSWEEPS % 2 == 1 else x
    del cz_
    return spec, raw, g, mask, out


def gpu_outputs(cfg, seed):
    d, sh, o, c, r, cx, cy, cz, al, cl = cfg
    spec, raw, g, a, mask = fixture_input(cfg, seed)
    lib = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / ref_configs.key(cfg) / "libref.so"))
    u3 = ctypes.c_uint * 3
    block = (8, 4, 2) if d == 3 else (8, 4, 1)
    gb = tuple(-(-g.threads[i] // block[i]) for i in range(3))
    out = np.empty_like(a)
    m = np.zeros(1) if mask is None else np.ascontiguousarray(mask)
    rc = lib.ref_sweeps(c.encode(), sh.encode(), ctypes.c_uint(r), ctypes.c_uint(d), al.encode(),
                        u3(*g.grid), u3(*block), u3(*gb), ctypes.c_uint(g.right_offset),
                        m.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(m.size if mask is not None else 0),
                        a.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p),
                        ctypes.c_uint(NSWEEPS))
    if rc != 0:
        raise RuntimeError("ref_sweeps failed (%d) for %s" % (rc, ref_configs.key(cfg)))
    return spec, raw, g, mask, out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--extra", action="store_true", help="the CPU-only sets of ref_configs.EXTRA")
    ap.add_argument("--out", default=str(HERE))
    a = ap.parse_args()
    outdir = Path(a.out)
    outdir.mkdir(parents=True, exist_ok=True)
    cfgs, seed0 = (ref_configs.EXTRA, 2000) if a.extra else (ref_configs.PARITY, 1000)
    with tempfile.TemporaryDirectory() as tmp:
        for i, cfg in enumerate(cfgs):
            seed = seed0 + i
            if a.gpu:
                spec, raw, g, mask, out = gpu_outputs(cfg, seed)
            else:
                spec, raw, g, mask, out = shim_outputs(cfg, seed, Path(tmp))
            np.savez_compressed(
                outdir / ("%s.npz" % ref_configs.key(cfg)), out=out, seed=seed, nsweeps=NSWEEPS,
                raw=np.array(raw), cfg=np.array([str(v) for v in cfg]),
                mask=np.zeros(0) if mask is None else mask, source=np.array("gpu" if a.gpu else "host-shim"))
            print("wrote", ref_configs.key(cfg))


if __name__ == "__main__":
    main()
