"""The reference's own host program (cuda/main.cpp, cuda/benchmark.cpp, cuda/primes.cpp, unmodified)
linked against the engine through launch_update_grid_shim.cpp: it must run and print the reference's
TSV report, in both its sweep and single-shape ("profile") modes."""

import subprocess
from pathlib import Path

import pytest

from oracle import ref_configs
from oracle.build_ref import SHIM_CONFIGS

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _exe(cfg):
    p = ROOT / "oracle" / "_ref" / ref_configs.key(cfg) / "bench_tcs"
    if not p.exists():
        pytest.skip("reference host program not built here")
    return p


def _rows(out: str):
    return [ln.split("\t") for ln in out.splitlines() if ln and not ln.startswith("#")]


def test_reference_host_program_sweep_2d():
    """Sweep mode (13 arguments).  The reference's single-shape ("profile") modes cannot be used:
    cuda/main.cpp:74-86 never parses the grid-size arguments in those modes, so the grid stays
    uninitialised and cuda/benchmark.cpp:600-609 rejects it."""
    exe = _exe(SHIM_CONFIGS[0])
    out = subprocess.run([str(exe), "Box", "2D", "1", "Jacobi", "Row", "None", "0", "0.002", "1", "1", "1024", "1024"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    assert "#xthreads\tythreads\tzthreads\tPerf [Flop/s]" in out.stdout
    rows = _rows(out.stdout)
    assert len(rows) == 464, out.stderr  # every 2D block shape at a 1024-thread limit
    for r in rows:
        iterations = int(r[7])
        assert iterations >= 1 and (iterations + 1) & iterations == 0, out.stderr  # 2^k - 1 launches
        assert float(r[5]) > 1e8


def test_reference_host_program_sweep_3d():
    exe = _exe(SHIM_CONFIGS[1])
    out = subprocess.run([str(exe), "Star", "3D", "4", "Variable", "Row", "Read", "16", "0.002", "2", "2", "1",
                          "128", "128", "128"], capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stderr
    rows = _rows(out.stdout)
    assert len(rows) > 100, out.stderr  # every block shape up to maxPotentialBlockSize
    assert all(int(r[7]) > 0 and float(r[5]) > 0 for r in rows), out.stderr
