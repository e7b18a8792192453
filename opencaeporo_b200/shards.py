"""Multi-GPU plumbing of the flash: independent cell shards, one process per
GPU. The flash has no cross-cell exchange, so ranks share nothing on the
data path; the process group only lines ranks up around timed regions and
takes the maximum of their device times (a rank's time is its own shard's
flash time; the job's time is the slowest rank's)."""
from __future__ import annotations

import datetime
import os


def env():
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 300):
    """Joins the process group when the job has more than one rank; returns
    the world size. With NCCL the rank's device must be set first."""
    import torch.distributed as dist
    world, rank, local = env()
    if world > 1 and not dist.is_initialized():
        kw = {}
        if backend == "nccl":
            import torch
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return world


def shard_seed(base_seed: int, rank: int) -> int:
    """Seed of rank's shard: every rank flashes its own cells (weak scaling)."""
    return base_seed + rank


def barrier():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.barrier()


def max_over_ranks(values, device=None):
    """Element-wise maximum of a list of floats over all ranks (identity on
    one rank)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized():
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def finalize():
    import torch.distributed as dist
    if dist.is_initialized():
        dist.barrier()
        dist.destroy_process_group()
