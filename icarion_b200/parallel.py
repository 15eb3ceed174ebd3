"""Multi-GPU decomposition of the batch step (one process per GPU).

Without space charge the ions are independent: each ion's Philox stream is
keyed on its global id, so a contiguous shard of ions per rank advances
exactly as it would in a single process.  The only exchange is the
per-snapshot sum of the ensemble moments (ICB_N_MOMENTS doubles per
ensemble) — one small all-reduce over NCCL (or gloo for CPU tests).

With space charge every step has one exchange: each rank exports its ions'
(x, y, z, q), an all-gather gives every rank all of them, and each rank's
solve deposits and pairs with every ion but computes the field of its own
(SpaceChargeExchange).  The mesh solve is repeated on every rank; the
particle-particle gather, the largest part, is split.
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


class SpaceChargeExchange:
    """Per-step exchange of the ranks' ions for a sharded space-charge solve.

    Every rank holds a buffer of world x n_max rows of (x, y, z, q) float64
    on its device; ``step()`` exports this rank's ions into its row block
    (rows beyond its own ions keep q = 0), all-gathers the blocks and hands
    the whole list to the handle with this rank's block as the skip range.
    Call it before every step (``sim.advance(1)``): the positions are those
    the step starts from.  The handle must launch on torch's current stream
    (``sim.set_stream``) so that the export, the collective and the step
    are ordered."""

    def __init__(self, sim, n_own: int, n_max: int, group=None):
        import torch
        import torch.distributed as dist
        self.sim, self.n_own, self.n_max, self.group = sim, int(n_own), int(n_max), group
        if self.n_own > self.n_max:
            raise ValueError("n_own exceeds n_max")
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        backend = dist.get_backend(group) if dist.is_initialized() else "none"
        dev = torch.device("cuda", torch.cuda.current_device()) if backend in ("nccl", "none") else torch.device("cpu")
        self.local = torch.zeros((self.n_max, 4), dtype=torch.float64, device=dev)
        self.all = torch.zeros((self.world * self.n_max, 4), dtype=torch.float64, device=dev)

    def step(self) -> None:
        import torch.distributed as dist
        self.sim.spacecharge_export(self.local.data_ptr())
        if self.world > 1:
            dist.all_gather_into_tensor(self.all, self.local, group=self.group)
            peers, n = self.all, self.world * self.n_max
        else:
            peers, n = self.local, self.n_max
        self.sim.set_spacecharge_peers(peers.data_ptr(), n, self.rank * self.n_max, self.n_max)
