"""Replica bookkeeping for runs on several GPUs of one node (one process per GPU).

The sweep does not shard in this engine: the reference is single-GPU (cuda/benchmark.cpp:105) and
its grids are swept by one device.  N ranks therefore run N independent replicas of a workload,
with no collective on the data path.  The only cross-rank steps are the timing ones: a barrier on
each side of a timed region, the maximum of the ranks' device times, and the whole-job rate = the
work of all ranks over the slowest rank's time.  Every rank takes these steps in the same order.
The backend is NCCL on GPUs; the same calls run over gloo on the CPU.
"""

from __future__ import annotations

import datetime
import os


def rank_env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment (1, 0, 0 without one)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init_group(world: int, backend: str = "nccl", timeout_s: float = 120.0):
    """The process group of a run with world > 1 (None for a single process).  The short timeout
    turns a rank that never arrives into an error on the others instead of a hang."""
    if world <= 1:
        return None
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(x: float, dist, device: str = "cuda") -> float:
    """The largest of the ranks' values of x (x itself for a single process)."""
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, units_per_rank: float, ms_max: float) -> float:
    """Units per second of the whole job: every rank's units over the slowest rank's time."""
    return world * float(units_per_rank) / (float(ms_max) / 1e3)


def close_group(dist) -> None:
    """Final barrier and teardown (every rank calls it, rank 0 included, before reporting)."""
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
