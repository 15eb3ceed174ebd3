"""Multi-GPU decomposition of the batch step (one process per GPU).

Without space charge the ions are independent: each ion's Philox stream is
keyed on its global id, so a contiguous shard of ions per rank advances
exactly as it would in a single process.  The only exchange is the
per-snapshot sum of the ensemble moments (ICB_N_MOMENTS doubles per
ensemble) — one small all-reduce over NCCL (or gloo for CPU tests).
"""
from __future__ import annotations

import numpy as np


def shard_range(n_total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous balanced split: rank r owns [begin, end)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, rem = divmod(n_total, world)
    begin = rank * base + min(rank, rem)
    return begin, begin + base + (1 if rank < rem else 0)


def shard_offsets(ens_offsets: np.ndarray, begin: int, end: int) -> np.ndarray:
    """Clip global ensemble offsets to the shard [begin, end), re-based at 0."""
    off = np.clip(np.asarray(ens_offsets, dtype=np.int64), begin, end) - begin
    return off.astype(np.uint64)


def allreduce_moments(mom: np.ndarray, group=None) -> np.ndarray:
    """Sum per-ensemble moments over all ranks with torch.distributed."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return mom
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(mom, dtype=np.float64)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def max_over_ranks(x: float, group=None) -> float:
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return x
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
