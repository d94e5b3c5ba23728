"""Host-side plumbing for one process per GPU (torch.distributed).

The particle filter does not shard in this library: N GPUs run N independent
replica filters (weak scaling).  The only cross-rank steps are the barrier
around a timed region and the max over ranks of the measured times, which
this module keeps in one place so that the CPU tests can exercise them with
the gloo backend.
"""
from __future__ import annotations

import datetime
import os


def world_info() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0):
    """Initialise the default process group from the environment (rendezvous
    at MASTER_ADDR / MASTER_PORT); returns torch.distributed, or None for a
    single process."""
    world, _, _ = world_info()
    if world <= 1:
        return None
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def sync_all(dist, device=None):
    """Barrier across ranks with the local device drained on both sides."""
    import torch
    if device is not None and device.type == "cuda":
        torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    if device is not None and device.type == "cuda":
        torch.cuda.synchronize(device)


def max_over_ranks(values, dist, device=None):
    """Element-wise max of a list of floats over all ranks."""
    if dist is None:
        return [float(v) for v in values]
    import torch
    dev = device if (device is not None and device.type == "cuda") else torch.device("cpu")
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def weak_scaling_rate(world: int, units_per_rank: float, seconds: float) -> float:
    """Whole-job throughput: every rank processed units_per_rank in at most
    `seconds` (the max over ranks)."""
    return world * units_per_rank / seconds


def finish(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
