"""Process-group plumbing for running the path on several GPUs of one node.

The MTTKRP of one tensor does not shard here: every rank runs its own replica
(one process per GPU, launched by torchrun) and the only communication is
timing bookkeeping -- a barrier around the timed region and the maximum of the
ranks' times.  Independent objects (the tensors of a batched CPD) are split
between ranks with `shard`, with no data exchange at all.  The backend is
NCCL on GPUs; the same functions run on the gloo backend on CPU.
"""
from __future__ import annotations

import datetime
import os


def setup(backend: str = "nccl", timeout_s: int = 600):
    """Reads RANK / WORLD_SIZE / LOCAL_RANK, selects the GPU (NCCL) and joins
    the process group when there is more than one rank.  Returns
    (rank, world, local_rank)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if backend == "nccl":
        import torch
        torch.cuda.set_device(local if world > 1 else 0)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """The largest of the ranks' values (every rank gets it)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(n_items: int, rank: int, world: int) -> range:
    """The contiguous share of n_items objects that rank `rank` of `world`
    processes: the first n_items % world ranks take one object more."""
    base, extra = divmod(int(n_items), int(world))
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def shutdown(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
