"""One process per GPU, each solving its own share of the job (weak scaling:
the EFIE path has no exchange step).  A sweep of incidences is split into
disjoint contiguous shares (``shard``), one per rank; each rank assembles and
factors its own Z and solves its share.  The only collectives are the timing
barrier, the max-over-ranks reduction of the device-timed interval and, after
the timed region, the gather of the per-incidence results to rank 0
(``gather_to_rank0``); rank 0 reports the whole-job rate."""
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


def shard(total: int, ws: int, rank: int) -> tuple[int, int]:
    """(start, count) of rank's contiguous share of `total` units: balanced,
    the first total % ws ranks take one more."""
    if ws < 1 or not (0 <= rank < ws) or total < 0:
        raise ValueError(f"bad shard request: total={total}, ws={ws}, rank={rank}")
    base, extra = divmod(total, ws)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def gather_to_rank0(x, device=None):
    """Concatenate every rank's 1-D float64 array in rank order on rank 0
    (None on the other ranks).  Shares may differ in length.  device: the CUDA
    device for NCCL, None for CPU tensors with gloo."""
    import numpy as np
    ws, rank, _ = replica_env()
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    if ws == 1:
        return a.copy()
    import torch
    import torch.distributed as dist
    n = torch.tensor([a.size], dtype=torch.int64, device=device)
    sizes = [torch.zeros_like(n) for _ in range(ws)]
    dist.all_gather(sizes, n)
    sizes = [int(t.item()) for t in sizes]
    m = max(sizes)
    buf = torch.zeros(m, dtype=torch.float64, device=device)
    buf[:a.size] = torch.from_numpy(a).to(buf.device)
    parts = [torch.zeros_like(buf) for _ in range(ws)]
    dist.all_gather(parts, buf)
    if rank != 0:
        return None
    return np.concatenate([p[:s].cpu().numpy() for p, s in zip(parts, sizes)])


def finalize() -> None:
    ws, _, _ = replica_env()
    if ws > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
