"""Benchmark of the B200 stencil engine (one JSON line on rank 0).

Default workload: 3D Star Variable stencil, range 4 (25 points), FP64, 512^3 grid, Read alignment to
16 points, seeded synthetic data (numpy default_rng; mask N(0,1) normalised to sum 1, values
U[0,1)).  A step is one sweep of the whole grid; `value` is the whole-job GLup/s (interior points
x steps / device time, max over ranks), with both 1 GiB buffers resident in HBM (inputs larger than
L2, so no flush is needed between sweeps).  `e2e` runs the reference's job shape through the C
ABI's host-buffer call (tcs_sweep_host_jobs): each job uploads the grid from pinned memory, runs
the workload's sweeps and downloads the result; --e2e-steps jobs rotate over 3 device slots so
uploads, sweeps and downloads of different jobs overlap (`serial_value`: the same jobs on one
slot), timed with CUDA events joined across the slots' streams.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Multi-GPU: the stencil does not shard in this engine (replicas only); each rank runs the same
workload on its own GPU and `value` sums the ranks' work over the slowest rank's time.
--impl reference times the reference's own arithmetic on the host cores: the CPU restatement of
the reference kernel (OpenMP, all host threads), the same metric and workload.
"""

from __future__ import annotations

import argparse
import json
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FALLBACK_HBM_GBS = 6650.0
# Nominal FP64 FMA peak: 148 SMs x 64 FMA/clk x 2 flops x 1.965 GHz.
FP64_PEAK_FLOPS = 148 * 64 * 2 * 1.965e9


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region.

    NVML is polled every ~5 ms from a thread (the device is matched by UUID); when NVML is not
    usable, `nvidia-smi --query-gpu ... -lms 200` is read instead."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index: int):
        self.index = index
        self.sm, self.smax, self.reasons = [], [], set()
        self.stop_flag = threading.Event()
        self.thread = None
        self.proc = None
        self.nvml = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.index).uuid)
        for cand in (uuid, "GPU-" + uuid):
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByUUID(cand)
            except Exception:
                continue
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = (nv, h)
            self.smax.append(float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)))
            getr = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons

            def poll():
                while not self.stop_flag.is_set():
                    try:
                        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                        bits = int(getr(h))
                        for bit, name in self.REASONS.items():
                            if bits & bit:
                                self.reasons.add(name)
                    except Exception:
                        pass
                    time.sleep(0.005)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        fields = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                  "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + fields,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def read():
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for line in self.proc.stdout:
                parts = [q.strip() for q in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    self.sm.append(float(parts[1]))
                    self.smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        self.reasons.add(name)

        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()

    def stop(self) -> dict:
        self.stop_flag.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": max(self.smax) if self.smax else None,
                    "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": max(self.smax) if self.smax else None,
                "reasons": sorted(self.reasons), "samples": len(self.sm),
                "source": "nvml" if self.nvml else "nvidia-smi"}


def _dist():
    """(world size, rank, local rank) from the launcher's environment (1, 0, 0 without one); read
    here without importing the engine, which the reference arm must not load."""
    import os

    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _traffic(workload: str):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text()).get(workload)
        if d:
            return d.get("dram_bytes_per_launch")
    return None


def cpu_baseline(w, spec, geom, a, mask, n: int, got=None) -> tuple[dict, dict | None]:
    """The oracle's OpenMP loop (all host threads) runs the same n ping-pong sweeps of the same
    grid that the GPU ran (warm-up and timed sweeps), from the same input.  Its time is the CPU
    baseline; its result is the checker of the GPU's (``got``): every point, bit for bit."""
    import numpy as np

    import oracle as O

    ospec = O.make_spec(spec.dimension, spec.neighbourhood, spec.orientation, spec.coefficients, spec.range,
                        spec.cx, spec.cy, spec.cz, spec.alignment, spec.cl_size)
    x = np.array(a, copy=True)
    y = np.array(a, copy=True)
    threads = O.max_threads()
    t0 = time.perf_counter()
    for _ in range(n):
        O.cpu_sweep(ospec, x, y, geom.right_offset, mask, threads=threads)
        x, y = y, x
    dt = time.perf_counter() - t0
    glups = geom.interior_points * n / dt / 1e9
    base = {"value": glups, "unit": "GLup/s", "cores": threads, "kind": "port",
            "sample": "%d full sweeps of the %s grid (%.1f s, OpenMP over rows, x innermost): the sweeps the GPU "
                      "ran, from the same input" % (n, "x".join(str(v) for v in w.grid[:w.spec.dimension]), dt)}
    parity = None
    if got is not None:
        same = bool(np.array_equal(got, x))
        diff = 0.0 if same else float(np.nanmax(np.abs(got.astype(np.float64) - x.astype(np.float64))))
        parity = {"equal": same, "sweeps": n, "points": "every point of both grids (interior, border, padding)",
                  "max_abs_diff": diff, "checker": "oracle OpenMP loop (same per-output term order)"}
    return base, parity


def reference_gpu_timing(w, geom, steps: int = 20) -> dict | None:
    """The reference's own generated kernel (built by oracle/build_ref.py for sm_100a) on this GPU."""
    import ctypes

    from oracle import ref_configs

    if not w.reference:
        return None
    (cx, cy, cz), block = w.reference
    s = w.spec
    cfg = (s.dimension, s.neighbourhood, s.orientation, s.coefficients, s.range, cx, cy, cz, s.alignment, s.cl_size)
    lib_path = ROOT / "oracle" / "_ref" / ref_configs.key(cfg) / "libref.so"
    if not lib_path.exists():
        return None
    rspec = s.replace(cx=cx, cy=cy, cz=cz)
    g = rspec.geometry(*w.grid)
    lib = ctypes.CDLL(str(lib_path))
    u3 = ctypes.c_uint * 3
    gb = tuple(max(1, -(-g.threads[i] // block[i])) for i in range(3))
    import numpy as np

    m = w.make_mask()
    mm = np.zeros(1) if m is None else np.ascontiguousarray(m)
    ms = ctypes.c_float()
    rc = lib.ref_time(ctypes.c_uint(s.dimension), u3(*g.grid), u3(*block), u3(*gb), ctypes.c_uint(g.right_offset),
                      mm.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint(0 if m is None else mm.size),
                      ctypes.c_uint(3), ctypes.c_uint(steps), ctypes.byref(ms))
    if rc != 0:
        return None
    glups = g.interior_points * steps / (ms.value / 1e3) / 1e9
    return {"value": glups, "unit": "GLup/s", "kernel": "reference generated updateGrid (nvcc -arch=sm_100a)",
            "coarsening": [cx, cy, cz], "block": list(block)}


def run_ours(args) -> dict | None:
    import numpy as np
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    from threadcoarsenedstencilgenerator_b200 import replicas

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = replicas.init_group(world, "nccl")
    w = WORKLOADS[args.workload]
    spec = w.tuned_spec()
    launch = w.tuned_launch()
    geom = spec.geometry(*w.grid)
    st = tcs.Stencil(spec)
    mask = w.make_mask()
    if mask is not None:
        st.copy_mask(mask)
    a = w.make_input(geom)
    host = torch.from_numpy(a).pin_memory()
    x = host.to("cuda", non_blocking=False)
    y = x.clone()
    plan = st.plan(geom, launch)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        st.update_grid(geom, x, y, launch, stream)
        x, y = y, x
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    replicas.barrier(dist)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        st.update_grid(geom, x, y, launch, stream)
        x, y = y, x
    e1.record(stream)
    torch.cuda.synchronize()
    replicas.barrier(dist)
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    if st.device_status() != 0:
        raise RuntimeError("device status word set during the timed sweeps")
    # the state the timed sweeps left (warm-up + timed sweeps from the seeded input), for the check
    result = x.cpu().numpy() if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None
    ms_max = replicas.max_over_ranks(ms, dist)
    points = geom.interior_points
    value = replicas.whole_job_rate(world, points * args.steps, ms_max) / 1e9

    # 2D: the same sweeps with temporal blocking (two sweeps per pass over HBM; same bits)
    temporal = None
    if spec.dimension == 2 and world == 1:
        st.sweeps_tb2(geom, x, y, 2 * args.warmup, stream)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        nt = args.steps + (args.steps % 2)
        t0.record(stream)
        st.sweeps_tb2(geom, x, y, nt, stream)
        t1.record(stream)
        torch.cuda.synchronize()
        tb_ms = t0.elapsed_time(t1)
        if st.device_status() != 0:
            raise RuntimeError("device status word set during the temporally blocked sweeps")
        tb_glups = geom.interior_points * nt / (tb_ms / 1e3) / 1e9
        temporal = {"glups": tb_glups, "sweeps": nt, "ms_per_sweep": tb_ms / nt,
                    "vs_single_sweep_kernel": tb_glups / (geom.interior_points * args.steps / (ms / 1e3) / 1e9),
                    "method": "tcs_sweeps_tb2: two sweeps per pass over HBM, bit-identical results"}

    # e2e: the reference's job shape (upload a grid from pinned host memory, w.sweeps sweeps,
    # download the result) through the C ABI's host-buffer entry point, e2e_steps jobs per step.
    # Jobs rotate over 3 device slots with a stream each, so one job's upload, another's sweeps and
    # a third's download overlap; the serial figure runs the same jobs on one slot.  Device time
    # from CUDA events joined across the slots' streams, max over ranks.
    e2e_steps = max(1, args.e2e_steps)
    slots = min(3, e2e_steps)
    outs = [torch.empty_like(host).pin_memory() for _ in range(slots)]
    dev = [(x, y)] + [(torch.empty_like(x), torch.empty_like(x)) for _ in range(slots - 1)]
    jobs_in = [host] * e2e_steps
    jobs_out = [outs[j % slots] for j in range(e2e_steps)]

    def _e2e(nslot):
        torch.cuda.synchronize()
        replicas.barrier(dist)
        out_ = jobs_out if nslot > 1 else [outs[0]] * e2e_steps
        ms_ = st.sweep_host_jobs(geom, jobs_in, out_, w.sweeps, launch, dev=dev[:nslot])
        return replicas.whole_job_rate(world, points * w.sweeps * e2e_steps, replicas.max_over_ranks(ms_, dist)) / 1e9

    e2e_value = _e2e(slots)
    e2e_serial = _e2e(1)
    nbytes = host.numel() * host.element_size()

    ref_gpu = None
    cpu = None
    parity = None
    if rank == 0 and world == 1:
        ref_gpu = reference_gpu_timing(w, geom)
        if not args.no_cpu_baseline:
            cpu, parity = cpu_baseline(w, spec, geom, a, mask, args.warmup + args.steps, result)
    replicas.close_group(dist)
    if rank != 0:
        return None

    peak, peak_kind = _peaks()
    bytes_per_launch = 2 * spec.itemsize * points  # algorithmic: one read + one write per point
    achieved = bytes_per_launch / ((ms / args.steps) / 1e3) / 1e9
    traffic = _traffic(args.workload)
    line = {
        "metric": "GLup/s (FP64 stencil sweep, %s)" % w.name,
        "value": value,
        "unit": "GLup/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if spec.precision == "f64" else "f32",
        "data": "synthetic (numpy default_rng seed %d)" % w.seed,
        "config": {
            "workload": w.name, "grid": list(w.grid[:spec.dimension]), "neighbourhood": spec.neighbourhood,
            "coefficients": spec.coefficients, "range": spec.range, "alignment": spec.alignment,
            "cl_size": spec.cl_size, "coarsening": list(spec.coarsening), "block": list(plan.block),
            "variant": plan.variant, "loader": plan.loader, "segments": plan.grid_blocks[-1 if spec.dimension == 3 else 1],
            "parallelism": "replicas" if world > 1 else "single-gpu",
            "l2": "inputs larger than L2 (2 x %.2f GiB)" % (nbytes / 2**30),
        },
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind
                     if peak_kind == "measured" else "fallback 6.65 TB/s",
                     "algorithmic_bytes_per_launch": bytes_per_launch},
        "e2e": {"value": e2e_value, "unit": "GLup/s", "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                "job": "upload grid, %d sweeps, download result (per step)" % w.sweeps, "steps": e2e_steps,
                "api": "tcs_sweep_host_jobs (C ABI, pinned host buffers)", "slots": slots,
                "serial_value": e2e_serial},
        "clocks": clocks,
        "cpu_baseline": cpu,
        "parity": None if parity is None else parity["equal"],
        "parity_check": parity,
        "reference_gpu": ref_gpu,
    }
    if temporal:
        line["temporal_blocking"] = temporal
    if world == 1 and not args.no_extras:
        del x, y, dev, outs, host, jobs_in, jobs_out
        line["configs"] = run_extras(args)
    return line


def run_config1(steps: int = 20, warmup: int = 3) -> dict:
    """2D Box Jacobi r1 (9-point mean) FP64 on 4096^2: the tuned single-sweep kernel and the
    two-sweeps-per-pass kernel (temporal blocking), each timed with CUDA events and checked against
    the oracle after the sweeps it ran."""
    import numpy as np
    import torch

    import oracle as O
    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    w = WORKLOADS["2d_box_jacobi_r1_4096"]
    spec = w.tuned_spec()
    launch = w.tuned_launch()
    geom = spec.geometry(*w.grid)
    st = tcs.Stencil(spec)
    a = w.make_input(geom)
    stream = torch.cuda.current_stream()
    peak, peak_kind = _peaks()
    ospec = O.make_spec(spec.dimension, spec.neighbourhood, spec.orientation, spec.coefficients, spec.range,
                        spec.cx, spec.cy, spec.cz, spec.alignment, spec.cl_size)
    out = {"workload": w.name, "coarsening": list(spec.coarsening), "block": list(launch.block),
           "variant": st.plan(geom, launch).variant}
    nt = steps + (steps % 2)
    for name, run in (("single_sweep", lambda u, v, k: st.sweeps(geom, u, v, k, launch, stream)),
                      ("temporal_blocking", lambda u, v, k: st.sweeps_tb2(geom, u, v, k, stream)),
                      ("temporal_blocking_strips", lambda u, v, k: st.sweeps_tb3(geom, u, v, k, None, stream))):
        x = torch.from_numpy(a).cuda()
        y = x.clone()
        run(x, y, 2 * warmup)
        torch.cuda.synchronize()
        x.copy_(torch.from_numpy(a))
        y.copy_(x)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        res = run(x, y, nt)
        e1.record(stream)
        torch.cuda.synchronize()
        if st.device_status() != 0:
            raise RuntimeError("device status word set during %s" % name)
        ms = e0.elapsed_time(e1)
        glups = geom.interior_points * nt / (ms / 1e3) / 1e9
        want = O.sweeps(ospec, a, nt, geom.right_offset, None, cpu_threads=0)
        bytes_per_lup = 16 if name == "single_sweep" else 8  # two sweeps per pass: 16 B per two updates
        achieved = glups * bytes_per_lup
        out[name] = {"glups": glups, "sweeps": nt, "ms_per_sweep": ms / nt,
                     "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                  "frac": achieved / peak, "peak_source": peak_kind,
                                  "algorithmic_bytes_per_lup": bytes_per_lup},
                     "parity": bool(np.array_equal(res.cpu().numpy(), want))}
        del x, y
    out["temporal_vs_single"] = out["temporal_blocking"]["glups"] / out["single_sweep"]["glups"]
    out["temporal_strips_vs_single"] = out["temporal_blocking_strips"]["glups"] / out["single_sweep"]["glups"]
    out["temporal_methods"] = {
        "temporal_blocking": "tcs_sweeps_tb2: tiles of 128 x 32 outputs loaded with their halo, two sweeps per pass",
        "temporal_blocking_strips": "tcs_sweeps_tb3 in 2D: strips marching along y through a TMA ring, stage 2 on "
                                    "stage 1's completed rows, two sweeps per pass"}
    out["roofline_note"] = ("single sweep: 16 B per lattice update (read + write); temporal blocking: 16 B per "
                            "two updates, so its HBM fraction counts 8 B per update")
    st.close()
    torch.cuda.empty_cache()
    return out


def run_extras(args) -> dict:
    """The other configurations of the workload list, each a compact record (single GPU): 2D Box
    Jacobi r1 (single sweep and temporal blocking), the 2D Box Variable r6 precision table, the
    batched uneven grids, and the learned autotuner live on held-out parameter sets."""
    import argparse as _ap

    import torch

    out = {}
    torch.cuda.empty_cache()
    out["config1_2d_box_jacobi_r1_4096"] = run_config1()
    torch.cuda.empty_cache()
    prec = run_precision(_ap.Namespace(workload="2d_box_var_r6_16384x8192", sweeps=200, period=20))
    out["config3_2d_box_var_r6_16384x8192"] = {"config": prec["config"], "precision": prec["precision"]}
    torch.cuda.empty_cache()
    b = run_batch(_ap.Namespace(workload="batch_3d_star_jacobi_r2_64", steps=5, warmup=3, e2e_steps=1,
                                no_cpu_baseline=True, gpus=1))
    out["config4_batch_3d_star_jacobi_r2_64"] = {"value": b["value"], "unit": b["unit"], "config": b["config"],
                                                 "roofline": b["roofline"], "batch": b["batch"]}
    torch.cuda.empty_cache()
    out["config5_autotune_live"] = run_autotune_live(3)
    return out


def run_autotune_live(n_sets: int) -> dict:
    """The learned tuner against the exhaustive sweep on the first n held-out parameter sets of the
    committed corpus (model top-5 timed, fallback rules as in production)."""
    from threadcoarsenedstencilgenerator_b200 import autotune as A

    cfg, X, y = A.load_corpus()
    hold, _ = A.split(cfg)
    m = A.CostModel.load()
    rows, rows_ref = [], []
    r = A.live(m, hold[:n_sets], log=lambda line: rows.append(line))
    # the same sets over the reference's whole block enumeration (cuda/primes.cpp: 464 shapes in 2D,
    # 2,723 in 3D): the model ranks shapes it never saw in training, the exhaustive sweep times all
    r_ref = A.live(m, hold[:n_sets], log=lambda line: rows_ref.append(line), space="reference")
    m.close()
    return {**r, "sets": [json.loads(q) for q in rows],
            "reference_space": {**r_ref, "sets": [json.loads(q) for q in rows_ref]}}


def run_precision(args) -> dict | None:
    """FP64 against the reduced-precision forms on one workload (single GPU), each from the same
    input for the workload's sweep count: plain FP32, compensated FP32, FP32 with FP64 defect
    correction every `period` sweeps, and (2D Box) the tensor-core sweep alone and with the same
    defect correction.  Errors are measured on the GPU against the engine's FP64 result (which is
    bit-identical to the reference kernel), three ways:

      per_sweep  one sweep of each raw form from the same input against one FP64 sweep -- the
                 accuracy of a single reduced-precision sweep;
      periods    the defect-corrected iterates against the FP64 iterate at every period boundary
                 (sweeps 20, 40, ...), including the boundaries before the iteration settles;
      final      after all sweeps.

    Relative errors: max_rel = max|a - b| / max|b|, rms_rel = ||a - b||_2 / ||b||_2 over the
    interior."""
    import numpy as np
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200.mixed import DefectCorrectedSweeps
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    torch.cuda.set_device(0)
    w = WORKLOADS[args.workload]
    spec = w.tuned_spec()
    launch = w.tuned_launch()
    geom = spec.geometry(*w.grid)
    mask = w.make_mask()
    n = args.sweeps or w.sweeps
    period = args.period
    a = w.make_input(geom)
    a32 = a.astype(np.float32)
    points = geom.interior_points
    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn):
        e0, e1 = ev(), ev()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1)

    def err(d):
        return {"max_rel": d["max_rel"], "rms_rel": d["rms_rel"]}

    # FP32 has a tuned shape of its own; it sweeps the FP64 geometry (partial coarsening tiles go
    # to the coarsening-1 fringe kernel, so the values do not depend on the shape)
    spec32 = w.tuned_spec("f32")
    launch32 = w.tuned_launch("f32")
    dc = DefectCorrectedSweeps(spec, launch, launch32=launch32, mask=mask, coarsening32=spec32.coarsening)
    s64, s32 = dc.s64, dc.s32
    s32c = tcs.Stencil(spec32.replace(precision="f32c"))
    if mask is not None:
        s32c.copy_mask(mask)
    tc_ok = spec.dimension == 2 and spec.neighbourhood == "Box" and spec.range <= 8
    dtc = DefectCorrectedSweeps(spec, launch, mask=mask, tensor_cores=True) if tc_ok else None

    x = torch.from_numpy(a).cuda()
    y = x.clone()
    x32 = torch.from_numpy(a32).cuda()
    y32 = x32.clone()

    # ---- per-sweep accuracy: one sweep of every form from the same input ----------------------
    s64.update_grid(geom, x, y, launch)
    per_sweep = {}
    s32.update_grid(geom, x32, y32, launch32)
    per_sweep["f32"] = err(s64.compare(geom, y32, y, "f32"))
    s32c.update_grid(geom, x32, y32, launch32)
    per_sweep["f32_compensated"] = err(s64.compare(geom, y32, y, "f32"))
    if dtc:
        dtc.s32.tc_update_grid(geom, x32, y32)
        per_sweep["tensor_cores"] = err(s64.compare(geom, y32, y, "f32"))
    torch.cuda.synchronize()

    def reset():
        x.copy_(torch.from_numpy(a))
        y.copy_(x)
        x32.copy_(torch.from_numpy(a32))
        y32.copy_(x32)

    # ---- throughput and final error over n sweeps ---------------------------------------------
    reset()
    s64.sweeps(geom, x, y, 3, launch)  # warm-up
    reset()
    ref, t64 = timed(lambda: s64.sweeps(geom, x, y, n, launch, stream))
    ref_final = ref.clone()
    forms = {}
    s32.sweeps(geom, x32, y32, 3, launch32)
    reset()
    r, t = timed(lambda: s32.sweeps(geom, x32, y32, n, launch32, stream))
    forms["f32"] = {"ms": t, **err(s64.compare(geom, r, ref_final, "f32")), "variant": s32.plan(geom, launch32).variant}
    s32c.sweeps(geom, x32, y32, 3, launch32)
    reset()
    r, t = timed(lambda: s32c.sweeps(geom, x32, y32, n, launch32, stream))
    forms["f32_compensated"] = {"ms": t, **err(s64.compare(geom, r, ref_final, "f32")),
                                "variant": s32c.plan(geom, launch32).variant}
    work = {"sx": torch.empty_like(x), "r": torch.zeros(geom.shape, dtype=torch.float32, device="cuda"),
            "e0": torch.zeros(geom.shape, dtype=torch.float32, device="cuda"),
            "e1": torch.zeros(geom.shape, dtype=torch.float32, device="cuda")}
    xm = torch.from_numpy(a).cuda()
    dc.run(geom, xm, 2, period, stream, work)  # warm-up
    xm.copy_(torch.from_numpy(a))
    (xm, res), t = timed(lambda: dc.run(geom, xm, n, period, stream, work))
    forms["f32_defect_corrected"] = {"ms": t, **err(s64.compare(geom, xm, ref_final, "f64")),
                                     "fp64_sweeps": res.fp64_sweeps, "fp32_sweeps": res.fp32_sweeps,
                                     "fused": dc.fused}
    xt = None
    if dtc:
        xt = torch.from_numpy(a).cuda()
        dtc.run(geom, xt, 2, period, stream, work)  # warm-up (Toeplitz operands, tensor maps)
        xt.copy_(torch.from_numpy(a))
        (xt, rtc), t = timed(lambda: dtc.run(geom, xt, n, period, stream, work))
        forms["tensor_cores_defect_corrected"] = {"ms": t, **err(s64.compare(geom, xt, ref_final, "f64"))}
        xs = torch.from_numpy(a32).cuda()
        ys = xs.clone()
        dtc.s32.tc_update_grid(geom, xs, ys)

        def tc_sweeps():
            u, v = xs, ys
            for _ in range(n):
                dtc.s32.tc_update_grid(geom, u, v)
                u, v = v, u
            return u

        r, t = timed(tc_sweeps)
        forms["tensor_cores"] = {"ms": t, **err(s64.compare(geom, r, ref_final, "f32"))}
        if dtc.s32.device_status() != 0:
            raise RuntimeError("device status word set during the tensor-core sweeps")
        del xs, ys

    # ---- defect-corrected iterates at every period boundary -----------------------------------
    periods = {"f32_defect_corrected": []}
    if dtc:
        periods["tensor_cores_defect_corrected"] = []
    reset()
    xm.copy_(torch.from_numpy(a))
    if xt is not None:
        xt.copy_(torch.from_numpy(a))
    done = 0
    cur = x
    while done < n:
        k = min(period, n - done)
        nxt = y if cur is x else x
        cur = s64.sweeps(geom, cur, nxt, k, launch, stream)
        dc.run(geom, xm, k, period, stream, work)
        periods["f32_defect_corrected"].append({"sweep": done + k, **err(s64.compare(geom, xm, cur, "f64"))})
        if xt is not None:
            dtc.run(geom, xt, k, period, stream, work)
            periods["tensor_cores_defect_corrected"].append({"sweep": done + k,
                                                             **err(s64.compare(geom, xt, cur, "f64"))})
        done += k
    for name, rows in periods.items():
        forms[name]["max_rel_over_periods"] = max(q["max_rel"] for q in rows)

    glups = lambda ms: points * n / (ms / 1e3) / 1e9  # noqa: E731
    for f in forms.values():
        f["glups"] = glups(f["ms"])
        f["speedup_vs_f64"] = t64 / f["ms"]
    # FP64 is bound by the FP64 pipe on long stencils: 2S-1 flops per point (cuda/benchmark.cpp:76-81)
    flops = spec.flops_per_update * points * n / (t64 / 1e3)
    return {
        "metric": "GLup/s (%s, %d sweeps, FP32 sweeps with FP64 defect correction every %d)" % (w.name, n, period),
        "value": glups(forms["f32_defect_corrected"]["ms"]), "unit": "GLup/s", "n_gpus": 1, "steps": n, "warmup": 3,
        "ms_per_step": forms["f32_defect_corrected"]["ms"] / n, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (numpy default_rng seed %d)" % w.seed,
        "config": {"workload": w.name, "grid": list(w.grid[:spec.dimension]), "coarsening": list(spec.coarsening),
                   "block": list(launch.block), "variant": launch.variant, "period": period,
                   "f32_coarsening": list(dc.spec32.coarsening), "f32_block": list(launch32.block),
                   "f32_chunk": launch32.chunk},
        "precision": {
            "f64": {"glups": glups(t64), "ms": t64, "tflops": flops / 1e12,
                    "fp64_pipe_frac_nominal": flops / FP64_PEAK_FLOPS},
            **forms,
            "per_sweep": per_sweep,
            "periods": periods,
            "error_definition": "max_rel = max|a-b| / max|b|, rms_rel = ||a-b||_2 / ||b||_2 over the interior, "
                                "b = FP64 result after the same sweeps from the same input",
        },
    }


def _batch_cpu(w, spec, geoms, arrs, budget_s: float, threads: int):
    """The oracle's OpenMP loop over the batch's grids, one after another, until the budget is
    spent (whole batch sweeps); returns (GLup/s, batch sweeps done, seconds)."""
    import numpy as np

    import oracle as O

    ospec = O.make_spec(spec.dimension, spec.neighbourhood, spec.orientation, spec.coefficients, spec.range,
                        spec.cx, spec.cy, spec.cz, spec.alignment, spec.cl_size)
    outs = [np.array(a, copy=True) for a in arrs]
    points = sum(g.interior_points for g in geoms)
    t0 = time.perf_counter()
    n = 0
    while True:
        for g, a, o in zip(geoms, arrs, outs):
            O.cpu_sweep(ospec, a, o, g.right_offset, None, threads=threads)
        n += 1
        if time.perf_counter() - t0 > budget_s or n >= 200:
            break
    dt = time.perf_counter() - t0
    return points * n / dt / 1e9, n, dt


def run_batch(args) -> dict | None:
    """Batched uneven grids: all grids swept by one persistent launch per sweep, the workload's
    sweeps captured in one CUDA graph; a step is one replay of that graph.  Beside it: the same
    sweeps as one launch per grid (plain stream launches, and captured in a graph too), and the
    batched launches without a graph.  FP64 is the headline; FP32 is measured the same way."""
    import numpy as np
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs
    from threadcoarsenedstencilgenerator_b200.batch import BatchedSweeps
    from threadcoarsenedstencilgenerator_b200.workloads import BATCH_WORKLOADS

    from threadcoarsenedstencilgenerator_b200 import replicas

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = replicas.init_group(world, "nccl")
    w = BATCH_WORKLOADS[args.workload]
    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    results = {}
    line_parts = {}
    for prec in ("f64", "f32"):
        spec = w.spec.replace(precision=prec)
        st = tcs.Stencil(spec)
        geoms = w.geometries(spec)
        arrs = w.make_inputs(geoms, np.float64 if prec == "f64" else np.float32)
        hosts = [torch.from_numpy(a).pin_memory() for a in arrs]
        xs = [h.to("cuda") for h in hosts]
        ys = [x.clone() for x in xs]
        launch = w.tuned_launch(prec)
        bt = BatchedSweeps(st, geoms, xs, ys, launch)
        plan = bt.plan()
        points = sum(g.interior_points for g in geoms)
        n = w.sweeps
        bt.capture(n)
        for _ in range(args.warmup):
            bt.replay(stream)
        torch.cuda.synchronize()
        main = prec == "f64"
        if main:
            sampler = ClockSampler(local)
            sampler.start()
            replicas.barrier(dist)
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        for _ in range(args.steps):
            bt.replay(stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if main:
            replicas.barrier(dist)
            clocks = sampler.stop()
        if st.device_status() != 0:
            raise RuntimeError("device status word set during the timed sweeps")
        # comparisons (per batch sweep)
        reps = max(1, min(10, args.steps // 5))
        ms_batched_nograph = timed(lambda: bt.sweeps(n, stream), reps) / n
        ms_separate = timed(lambda: bt.sweeps(n, stream, separate=True), reps) / n
        bt.capture(n, separate=True)
        ms_separate_graph = timed(lambda: bt.replay(stream), reps) / n
        bt.capture(n)
        per_sweep = ms / args.steps / n
        glups = lambda t: points / (t / 1e3) / 1e9  # noqa: E731
        results[prec] = {
            "glups": world * glups(per_sweep), "ms_per_sweep": per_sweep,
            "batched_graph_glups": glups(per_sweep), "batched_launches_glups": glups(ms_batched_nograph),
            "separate_launches_glups": glups(ms_separate), "separate_launches_graph_glups": glups(ms_separate_graph),
            "speedup_vs_separate_launches": ms_separate / per_sweep,
            "speedup_vs_separate_launches_graph": ms_separate_graph / per_sweep,
            "block": list(plan.block), "ctas": plan.grid_blocks[0], "loader": plan.loader, "chunk": plan.chunk,
            "depth": plan.depth,
        }
        if main:
            ms_max = replicas.max_over_ranks(ms, dist)
            # e2e: every step uploads all grids from pinned memory, replays the graph, downloads
            outs = [torch.empty_like(h).pin_memory() for h in hosts]
            e2e_steps = max(1, args.e2e_steps)
            torch.cuda.synchronize()
            f0, f1 = ev(), ev()
            f0.record(stream)
            for _ in range(e2e_steps):
                for h, x, y in zip(hosts, xs, ys):
                    x.copy_(h, non_blocking=True)
                    y.copy_(x)
                res = bt.replay(stream)
                for o, r in zip(outs, res):
                    o.copy_(r, non_blocking=True)
            f1.record(stream)
            torch.cuda.synchronize()
            te_max = replicas.max_over_ranks(f0.elapsed_time(f1), dist)
            nbytes = sum(h.numel() * h.element_size() for h in hosts)
            line_parts = {
                "ms_max": ms_max, "points": points, "nbytes": nbytes, "plan": plan, "clocks": clocks,
                "e2e": {"value": replicas.whole_job_rate(world, points * n * e2e_steps, te_max) / 1e9, "unit": "GLup/s",
                        "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                        "job": "upload %d grids, %d batched sweeps (graph), download results" % (len(geoms), n),
                        "steps": e2e_steps},
                "itemsize": spec.itemsize, "geoms": geoms, "arrs": arrs, "spec": spec,
            }
        bt.close()
        del xs, ys, hosts
        torch.cuda.empty_cache()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle as O

        threads = O.max_threads()
        v, nsw, dt = _batch_cpu(w, line_parts["spec"], line_parts["geoms"], line_parts["arrs"], 12.0, threads)
        cpu = {"value": v, "unit": "GLup/s", "cores": threads, "kind": "port",
               "sample": "%d sweeps of all %d grids (%.1f s, OpenMP restatement, grid after grid)" % (
                   nsw, w.n_grids, dt)}
    replicas.close_group(dist)
    if rank != 0:
        return None
    peak, peak_kind = _peaks()
    n = w.sweeps
    points = line_parts["points"]
    ms_max = line_parts["ms_max"]
    per_launch_ms = results["f64"]["ms_per_sweep"]
    bytes_per_launch = 2 * line_parts["itemsize"] * points
    achieved = bytes_per_launch / (per_launch_ms / 1e3) / 1e9
    plan = line_parts["plan"]
    return {
        "metric": "GLup/s (FP64 batched sweeps, %s)" % w.name,
        "value": replicas.whole_job_rate(world, points * n * args.steps, ms_max) / 1e9,
        "unit": "GLup/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (numpy default_rng seed %d)" % w.seed,
        "config": {"workload": w.name, "grids": w.n_grids, "sides": "log-uniform [%d, %d], multiples of %d" % (
                   w.side_range[0], w.side_range[1], w.multiple), "neighbourhood": w.spec.neighbourhood,
                   "coefficients": w.spec.coefficients, "range": w.spec.range,
                   "coarsening": list(w.spec.coarsening), "block": list(plan.block), "ctas": plan.grid_blocks[0],
                   "step": "one CUDA-graph replay of %d batched sweeps (one persistent launch per sweep)" % n,
                   "parallelism": "replicas" if world > 1 else "single-gpu",
                   "l2": "inputs larger than L2 (2 x %.2f GiB over all grids)" % (line_parts["nbytes"] / 2**30)},
        "gpu_launches": args.steps * n,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": _traffic(w.name), "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind
                     if peak_kind == "measured" else "fallback 6.65 TB/s",
                     "algorithmic_bytes_per_launch": bytes_per_launch},
        "e2e": line_parts["e2e"],
        "clocks": line_parts["clocks"],
        "cpu_baseline": cpu,
        "batch": results,
    }


def _workload_params():
    """The workload table, loaded from its file without importing the engine's package (the
    reference arm must not map libtcs.so)."""
    import importlib.util

    path = ROOT / "threadcoarsenedstencilgenerator_b200" / "workload_params.py"
    spec = importlib.util.spec_from_file_location("tcs_workload_params", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _oracle_shape(dimension: int, g) -> tuple:
    return (g.grid[1], g.grid[0]) if dimension == 2 else (g.grid[2], g.grid[1], g.grid[0])


def _oracle_points(dimension: int, g) -> int:
    e = g.elements
    return e[0] * e[1] * (e[2] if dimension == 3 else 1)


def run_reference(args) -> dict | None:
    """The reference's own stencil arithmetic on the host cores (oracle OpenMP restatement).  Only
    the oracle is loaded: the workload table comes from its plain-data file and the geometry from
    the oracle's restatement of cuda/benchmark.cpp:142-179."""
    import oracle as O

    world, rank, local = _dist()
    if rank != 0:
        return None
    P = _workload_params()
    if args.workload in P.BATCH:
        p = P.BATCH[args.workload]
        st = p["stencil"]
        ospec = O.make_spec(*st)
        sides = P.batch_sides(p["n_grids"], p["side_range"], p["multiple"], p["seed"])
        geoms = [O.geometry(ospec, *sd) for sd in sides]
        arrs = P.batch_inputs(p["seed"], [_oracle_shape(st[0], g) for g in geoms])
        points = sum(_oracle_points(st[0], g) for g in geoms)
        threads = O.max_threads()
        outs = [a.copy() for a in arrs]

        def batch_sweep():
            for g, a, o in zip(geoms, arrs, outs):
                O.cpu_sweep(ospec, a, o, g.right_offset, None, threads=threads)
            return [(o, a) for a, o in zip(arrs, outs)]

        for _ in range(args.warmup):
            pairs = batch_sweep()
            arrs, outs = [q for q, _ in pairs], [q for _, q in pairs]
        t0 = time.perf_counter()
        nsw = 0
        while nsw < args.steps and (nsw == 0 or time.perf_counter() - t0 < 20.0):
            pairs = batch_sweep()
            arrs, outs = [q for q, _ in pairs], [q for _, q in pairs]
            nsw += 1
        dt = time.perf_counter() - t0
        value = points * nsw / dt / 1e9
        return {
            "metric": "GLup/s (FP64 batched sweeps, %s)" % args.workload, "value": value, "unit": "GLup/s",
            "n_gpus": world, "steps": nsw, "warmup": args.warmup, "ms_per_step": dt * 1e3 / nsw,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (numpy default_rng seed %d)" % p["seed"],
            "config": {"workload": args.workload, "grids": p["n_grids"]}, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "GLup/s", "cores": threads, "kind": "port",
                             "sample": "%d sweeps of all %d grids, OpenMP restatement of the reference kernel, "
                                       "grid after grid" % (nsw, p["n_grids"])},
            "e2e": {"value": value, "unit": "GLup/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    p = P.SINGLE[args.workload]
    st = p["stencil"]
    ospec = O.make_spec(*st)
    geom = O.geometry(ospec, *p["grid"])
    right = geom.right_offset
    a = P.make_input(p["seed"], p["value_range"], _oracle_shape(st[0], geom))
    mask = P.make_mask(p["seed"], p["mask_kind"], st)
    out = a.copy()
    threads = O.max_threads()
    for _ in range(args.warmup):
        O.cpu_sweep(ospec, a, out, right, mask, threads=threads)
        a, out = out, a
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.cpu_sweep(ospec, a, out, right, mask, threads=threads)
        a, out = out, a
    dt = time.perf_counter() - t0
    value = _oracle_points(st[0], geom) * args.steps / dt / 1e9
    return {
        "metric": "GLup/s (FP64 stencil sweep, %s)" % args.workload, "value": value, "unit": "GLup/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (numpy default_rng seed %d)" % p["seed"],
        "config": {"workload": args.workload, "grid": list(p["grid"][:st[0]])}, "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "GLup/s", "cores": threads, "kind": "port",
                         "sample": "%d full sweeps of the grid, OpenMP restatement of the reference kernel" % args.steps},
        "e2e": {"value": value, "unit": "GLup/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_case(args) -> dict:
    """A few sweeps of a workload's tuned launch on a reduced grid (--grid) or on the first K grids
    of a batch (--grids), for profilers: a small case of the same kernel that an ncu capture
    finishes in a minute.  Keep each buffer above the L2 size (126 MB) so that DRAM counters
    stay meaningful.  --case tensor-cores / temporal select the tcgen05 FP32 sweep / the
    two-sweeps-per-pass kernel (2D); --case-launch one pipelined launch instead of the tuned one.
    One warm-up sweep (two for temporal) precedes the --steps sweeps, whose rate is reported from
    CUDA events ("glups"; 1-GPU case timing, not the bench line)."""
    import numpy as np
    import torch

    import threadcoarsenedstencilgenerator_b200 as tcs

    torch.cuda.set_device(0)
    P = _workload_params()
    if args.workload in P.BATCH:
        from threadcoarsenedstencilgenerator_b200.batch import BatchedSweeps
        from threadcoarsenedstencilgenerator_b200.workloads import BATCH_WORKLOADS

        w = BATCH_WORKLOADS[args.workload]
        spec = w.spec.replace(precision=args.case_precision)
        geoms = w.geometries(spec)
        arrs = w.make_inputs(geoms, np.float64 if args.case_precision == "f64" else np.float32)
        if args.grids:
            geoms, arrs = geoms[:args.grids], arrs[:args.grids]
        st = tcs.Stencil(spec)
        xs = [torch.from_numpy(v).cuda() for v in arrs]
        ys = [x.clone() for x in xs]
        bt = BatchedSweeps(st, geoms, xs, ys, w.tuned_launch(args.case_precision))
        bt.sweeps(args.steps)
        torch.cuda.synchronize()
        if st.device_status() != 0:
            raise RuntimeError("device status word set")
        plan = bt.plan()
        bt.close()
        return {"case": args.workload, "grids": len(geoms), "points": sum(g.interior_points for g in geoms),
                "sweeps": args.steps, "block": list(plan.block), "loader": plan.loader}
    from threadcoarsenedstencilgenerator_b200.workloads import WORKLOADS

    w = WORKLOADS[args.workload]
    spec = w.tuned_spec(args.case_precision).replace(precision=args.case_precision)
    launch = w.tuned_launch(args.case_precision)
    tb3_launch = None  # temporal-strips: the two-sweep kernel's block, chunk and CTA count
    if args.case_launch:
        case_spec, launch = case_launch(spec, args.case_launch)
        if args.case == "temporal-strips":
            tb3_launch = launch  # its thread tiles are its own: the parameter set keeps its coarsening
        else:
            spec = case_spec
    grid = tuple(args.grid) + (1,) * (3 - len(args.grid))
    geom = spec.geometry(*grid)
    st = tcs.Stencil(spec)
    m = w.make_mask()
    if m is not None:
        st.copy_mask(m)
    dt = torch.float64 if args.case_precision == "f64" else torch.float32
    x = torch.from_numpy(w.make_input(geom)).to("cuda", dtype=dt)
    y = x.clone()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def run(n):
        nonlocal x, y
        if args.case == "temporal":
            st.sweeps_tb2(geom, x, y, n)
            return
        if args.case == "temporal-strips":
            st.sweeps_tb3(geom, x, y, n, tb3_launch)
            return
        for _ in range(n):
            if args.case == "tensor-cores":
                st.tc_update_grid(geom, x, y)
            else:
                st.update_grid(geom, x, y, launch)
            x, y = y, x

    run(2 if args.case.startswith("temporal") else 1)  # warm-up (module load, first touch)
    torch.cuda.synchronize()
    e0.record(stream)
    run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if st.device_status() != 0:
        raise RuntimeError("device status word set")
    plan = st.plan_tb3(geom, tb3_launch) if args.case == "temporal-strips" else st.plan(geom, launch)
    ms = e0.elapsed_time(e1)  # CUDA events around the --steps sweeps after the warm-up
    return {"case": args.workload, "grid": list(grid), "points": geom.interior_points, "sweeps": args.steps,
            "kernel": args.case, "variant": plan.variant, "block": list(plan.block), "chunk": plan.chunk,
            "coarsening": [spec.cx, spec.cy, spec.cz], "shuffle": bool(launch.shuffle), "tmem": bool(launch.tmem),
            "glups": geom.interior_points * args.steps / (ms / 1e3) / 1e9 if ms > 0 else None}


def case_launch(spec, text: str):
    """(spec, Launch) of a pipelined launch written cx,cy,bx,by,chunk[,shuffle[,tmem[,ctas]]]: the
    profiling case of one point of the launch space instead of the tuned launch (ctas: the number
    of persistent CTAs, 0 = one wave)."""
    from threadcoarsenedstencilgenerator_b200.stencil import Launch

    v = [int(t) for t in text.split(",")]
    if len(v) not in (5, 6, 7, 8):
        raise SystemExit("--case-launch wants cx,cy,bx,by,chunk[,shuffle[,tmem[,ctas]]]")
    cx, cy, bx, by, ch = v[:5]
    spec = spec.replace(cx=cx, cy=cy, cz=1) if spec.dimension == 3 else spec.replace(cx=cx, cy=1)
    return spec, Launch(block=(bx, by, 1), variant="pipe", chunk=ch, shuffle=bool(v[5]) if len(v) > 5 else False,
                        tmem=bool(v[6]) if len(v) > 6 else False, segments=v[7] if len(v) > 7 else 0)


def check_world(gpus: int, world: int) -> str | None:
    """An error message when --gpus disagrees with the launcher's world size, else None.  bench.py
    runs one process per GPU: --gpus N > 1 needs N ranks from torch.distributed.run."""
    if gpus < 1:
        return "--gpus must be at least 1"
    if gpus != world:
        return ("--gpus %d but WORLD_SIZE is %d: launch one process per GPU, e.g. python -m "
                "torch.distributed.run --nnodes=1 --nproc-per-node %d --master-addr 127.0.0.1 bench.py --gpus %d"
                % (gpus, world, gpus, gpus))
    return None


def main(argv=None) -> int:
    P = _workload_params()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default=P.DEFAULT, choices=sorted(P.SINGLE) + sorted(P.BATCH))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline workload only (skip the other configurations' records)")
    ap.add_argument("--precision", default="f64", choices=["f64", "mixed"],
                    help="mixed: FP64 vs FP32 vs FP32 with FP64 defect correction on the workload")
    ap.add_argument("--sweeps", type=int, default=0, help="precision mode: sweeps (default: the workload's)")
    ap.add_argument("--period", type=int, default=20, help="precision mode: FP32 sweeps per FP64 defect")
    ap.add_argument("--grid", type=int, nargs="+", help="profiling case: --steps sweeps on this reduced grid")
    ap.add_argument("--grids", type=int, default=0, help="profiling case (batch): the first K grids")
    ap.add_argument("--case", default="sweep", choices=["sweep", "tensor-cores", "temporal", "temporal-strips"],
                    help="profiling case: which kernel")
    ap.add_argument("--case-precision", default="f64", choices=["f64", "f32"], help="profiling case: precision")
    ap.add_argument("--case-launch", default="", help="profiling case: pipelined launch "
                    "cx,cy,bx,by,chunk[,shuffle[,tmem[,ctas]]] instead of the tuned one")
    args = ap.parse_args(argv)
    args.warmup = max(3, args.warmup)
    err = check_world(args.gpus, _dist()[0])
    if err:
        print(err, file=sys.stderr)
        return 2
    if args.impl == "reference":
        line = run_reference(args)
    elif args.grid or args.grids:
        line = run_case(args)
    elif args.workload in P.BATCH:
        line = run_batch(args)
    elif args.precision == "mixed":
        line = run_precision(args)
    else:
        line = run_ours(args)
    if line is not None:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
