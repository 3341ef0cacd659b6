"""Multi-rank bookkeeping of the benchmark, run as gloo ranks on the CPU (no GPU).

The sweep does not shard, so N ranks are N replicas; what crosses ranks is the timing: barriers
around the timed region, the maximum of the ranks' times, and the whole-job rate over the
slowest rank.  These tests run that code as two processes over gloo, and check that a rank which
never joins turns into an error on the other one, not a hang.
"""

import argparse
import json
import os
import socket
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

from threadcoarsenedstencilgenerator_b200 import replicas

ROOT = Path(__file__).resolve().parents[1]

RANK_SCRIPT = textwrap.dedent("""
    import json, sys
    sys.path.insert(0, %(root)r)
    from threadcoarsenedstencilgenerator_b200 import replicas
    world, rank, local = replicas.rank_env()
    dist = replicas.init_group(world, "gloo", timeout_s=float(sys.argv[1]))
    replicas.barrier(dist)
    ms = 10.0 + 5.0 * rank          # this rank's device time for the timed region
    ms_max = replicas.max_over_ranks(ms, dist, device="cpu")
    rate = replicas.whole_job_rate(world, 1000.0, ms_max)
    replicas.close_group(dist)
    print(json.dumps({"rank": rank, "world": world, "ms_max": ms_max, "rate": rate}))
""")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(rank: int, world: int, port: int, timeout_s: float, script: str):
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
               RANK=str(rank), LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    return subprocess.Popen([sys.executable, "-c", script, str(timeout_s)], env=env, stdout=subprocess.PIPE,
                            stderr=subprocess.PIPE, text=True)


def test_two_gloo_ranks_report_the_slowest_rank():
    port = _free_port()
    script = RANK_SCRIPT % {"root": str(ROOT)}
    procs = [_launch(r, 2, port, 60.0, script) for r in range(2)]
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["ms_max"] == 15.0                       # max over ranks, the same on every rank
        assert o["rate"] == pytest.approx(2 * 1000.0 / 0.015)  # both ranks' work over the slowest time
    assert sorted(o["rank"] for o in outs) == [0, 1]


def test_rank_that_never_joins_is_an_error_not_a_hang():
    port = _free_port()
    script = RANK_SCRIPT % {"root": str(ROOT)}
    p = _launch(0, 2, port, 3.0, script)  # rank 1 is never started
    out, err = p.communicate(timeout=120)
    assert p.returncode != 0
    assert "rank" not in out


def test_single_process_needs_no_group(monkeypatch):
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.rank_env() == (1, 0, 0)
    assert replicas.init_group(1) is None
    assert replicas.max_over_ranks(7.5, None, device="cpu") == 7.5
    assert replicas.whole_job_rate(1, 500.0, 250.0) == 2000.0
    replicas.close_group(None)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    """Under torchrun the reference arm prints from rank 0; the other ranks exit without work."""
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = argparse.Namespace(workload="3d_star_var_r4_512", steps=3, warmup=3, gpus=2, e2e_steps=1,
                              no_cpu_baseline=True, impl="reference")
    assert bench.run_reference(args) is None
