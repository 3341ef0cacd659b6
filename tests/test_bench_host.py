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
