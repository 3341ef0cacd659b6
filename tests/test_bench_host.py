"""Host-side pieces of bench.py (no GPU): the roofline denominator, the per-launch DRAM traffic
table and the clock-event reason names."""

import json

import pytest

import bench
from threadcoarsenedstencilgenerator_b200.workloads import BATCH_WORKLOADS, WORKLOADS


def test_peak_is_the_measured_copy_when_present(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench._peaks() == (bench.FALLBACK_HBM_GBS, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6542.0, "bf16_tflops": 1590.0}))
    assert bench._peaks() == (6542.0, "measured")


def test_traffic_table_is_per_launch_and_near_the_algorithmic_bytes():
    """Each entry is one launch's ncu DRAM bytes; it must sit between the algorithmic bytes
    (one read and one write of every interior point, FP64) and 1.5 times them."""
    for name, entry in json.loads((bench.ROOT / "profiles" / "traffic.json").read_text()).items():
        traffic = entry["dram_bytes_per_launch"]
        assert bench._traffic(name) == traffic
        if name in WORKLOADS:
            w = WORKLOADS[name]
            spec = w.tuned_spec()
            points = spec.geometry(*w.grid).interior_points
        else:
            w = BATCH_WORKLOADS[name]
            points = sum(g.interior_points for g in w.geometries(w.spec))
        algorithmic = 16 * points
        assert algorithmic <= traffic <= 1.5 * algorithmic, name
    assert bench._traffic("no such workload") is None


@pytest.mark.parametrize("bit, name", [(0x4, "sw_power_cap"), (0x8, "hw_slowdown"), (0x20, "sw_thermal_slowdown"),
                                       (0x40, "hw_thermal_slowdown"), (0x80, "hw_power_brake_slowdown")])
def test_clock_event_reason_bits(bit, name):
    """NVML's clocks-event reason bits, by the names the rejection rule uses."""
    assert bench.ClockSampler.REASONS[bit] == name


def test_gpus_must_match_the_launchers_world_size():
    """--gpus N is one process per GPU: a mismatch with WORLD_SIZE is an error, not a silent
    single replica."""
    assert bench.check_world(1, 1) is None
    assert bench.check_world(4, 4) is None
    assert "WORLD_SIZE is 1" in bench.check_world(8, 1)
    assert bench.check_world(0, 1) is not None
    import subprocess
    import sys

    proc = subprocess.run([sys.executable, str(bench.ROOT / "bench.py"), "--gpus", "2", "--steps", "1"],
                          capture_output=True, text=True, env={**__import__("os").environ, "WORLD_SIZE": "1"})
    assert proc.returncode == 2 and "torch.distributed.run" in proc.stderr
    assert proc.stdout.strip() == ""


def test_reference_arm_loads_only_the_oracle():
    """bench.py --impl reference runs the oracle's OpenMP restatement: it must neither import the
    engine's package nor map libtcs.so (the workload table is read from its plain-data file)."""
    import subprocess
    import sys

    code = (
        "import sys, json; sys.path.insert(0, %r); import bench; "
        "rc = bench.main(['--impl', 'reference', '--workload', '2d_box_jacobi_r1_4096', '--steps', '2', "
        "'--warmup', '3']); "
        "maps = open('/proc/self/maps').read(); "
        "assert rc == 0; "
        "assert 'libtcs' not in maps, 'libtcs.so mapped'; "
        "assert not any(m.startswith('threadcoarsenedstencilgenerator_b200') for m in sys.modules), 'package imported'; "
        "assert 'liboracle' in maps"
    ) % str(bench.ROOT)
    proc = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-2000:]
    line = json.loads(proc.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2
    assert line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_workload_table_matches_the_engine_workloads():
    """The plain-data table and the engine's Workload objects describe the same runs."""
    import numpy as np

    P = bench._workload_params()
    for name, w in WORKLOADS.items():
        p = P.SINGLE[name]
        s = w.spec
        assert p["stencil"] == (s.dimension, s.neighbourhood, s.orientation, s.coefficients, s.range, s.cx, s.cy,
                                s.cz, s.alignment, s.cl_size)
        assert tuple(p["grid"]) == w.grid and p["sweeps"] == w.sweeps
        assert P.stencil_size(p["stencil"]) == s.stencil_size
        m = w.make_mask()
        pm = P.make_mask(p["seed"], p["mask_kind"], p["stencil"])
        assert (m is None and pm is None) or np.array_equal(m, pm)
    for name, w in BATCH_WORKLOADS.items():
        p = P.BATCH[name]
        assert P.batch_sides(p["n_grids"], p["side_range"], p["multiple"], p["seed"]) == w.sides()
