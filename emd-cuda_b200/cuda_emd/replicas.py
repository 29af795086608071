"""Replica runs over several GPUs: one process per GPU, each decomposing its
own batch of traces.  Traces never interact (the reference processes each
signal independently, kernels.py:6-10), so there is no collective on the data
path -- only a barrier around timed regions and the maximum of the ranks'
device times, from which the whole-job rate follows (weak scaling: fixed work
per rank).  The process group backend is NCCL on GPUs; the same code runs on
gloo for tests on the host."""
from __future__ import annotations

import datetime
import os


def rank_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(world: int, backend: str = "nccl", device=None, timeout_s: float = 120.0) -> None:
    """Join the process group (world > 1) with a short timeout, so ranks that
    wait for a missing peer fail instead of hanging."""
    if world <= 1:
        return
    import torch.distributed as dist
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None and backend == "nccl":
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)


def workload_seed(base: int, rank: int) -> int:
    """Each rank's own seeded batch (distinct data, same distribution)."""
    return base + 1000 * rank


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(seconds: float, world: int, device=None) -> float:
    """The largest of the ranks' timings (every rank gets it)."""
    if world <= 1:
        return float(seconds)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(seconds)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(traces_per_rank: int, steps: int, world: int, seconds_max: float) -> float:
    """Traces per second of the whole job: every rank's traces over the
    slowest rank's time."""
    return traces_per_rank * steps * world / seconds_max


def finish(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
