"""One process per GPU: the rank plumbing of multi-GPU runs.

The path has no data exchange: fields (framework x guest) and pose batches are
independent, so N ranks either compute N independent fields (weak scaling) or
split a list of fields between them.  The only collective is the max over
ranks of a device time.  Rendezvous is on 127.0.0.1; every rank takes the
same collective steps in the same order."""
from __future__ import annotations

import datetime
import os


def rank_info() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, local_rank: int, timeout_s: float = 300.0) -> None:
    """Join the process group (nccl: one GPU per rank; gloo: CPU tests)."""
    import torch
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    kwargs = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        torch.cuda.set_device(local_rank)
        kwargs["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, **kwargs)


def shard(items, rank: int, world: int) -> list:
    """Round-robin share of `items` for this rank (disjoint, covering)."""
    return list(items)[rank::world]


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (the time of a step: the slowest rank)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
