"""One process per GPU, each solving its own copy of the job (replicas, weak
scaling: the EFIE path has no exchange step).  The only collectives are the
timing barrier and the max-over-ranks reduction of the device-timed
interval; rank 0 reports the whole-job rate."""
from __future__ import annotations

import datetime
import os


def replica_env():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 300.0) -> None:
    """Join the process group when more than one rank runs (MASTER_ADDR /
    MASTER_PORT from the launcher; use 127.0.0.1)."""
    ws, _, _ = replica_env()
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def barrier() -> None:
    ws, _, _ = replica_env()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, device=None) -> float:
    """Max of a per-rank float over all ranks (device: the CUDA device for
    NCCL, None for a CPU tensor with gloo)."""
    ws, _, _ = replica_env()
    if ws == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, ms_max: float) -> float:
    """Whole-job units per second: every rank processed units_per_rank in at
    most ms_max milliseconds."""
    ws, _, _ = replica_env()
    return ws * units_per_rank / (ms_max / 1e3)


def finalize() -> None:
    ws, _, _ = replica_env()
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
