"""Multi-rank decomposition on CPU: two gloo ranks each advance their shard of
the ions (ion ids offset by the shard start, so each ion keeps its Philox
stream) and all-reduce the per-snapshot moments; the result must equal one
process advancing all ions.  The advancing is done by the CPU oracle with the
product's null-collision scheme, which is exactly what each GPU rank runs."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

N_IONS, STEPS, SNAP = 600, 400, 100


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_path: str) -> None:
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    for p in (str(root), str(root / "oracle"), str(root / "tests")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import oracle as orc
    from helpers import config0_ensemble, config0_ions, oracle_state
    from icarion_b200 import parallel

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        full = oracle_state(config0_ions(N_IONS))
        b, e = parallel.shard_range(N_IONS, rank, world)
        shard = {k: np.ascontiguousarray(v[b:e]) for k, v in full.items()}
        r = orc.run(config0_ensemble(), shard, STEPS, integrator=0, collision=2, seed=123, first_id=b,
                    snap_every=SNAP, ref_step=SNAP)
        mom = parallel.allreduce_moments(r["moments"])
        counts = parallel.allreduce_moments(np.array([r["candidates"], r["collisions"]], dtype=np.float64))
        if rank == 0:
            np.savez(out_path, moments=mom, counts=counts)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_equal_one_process(tmp_path):
    from helpers import config0_ensemble, config0_ions, oracle_state
    import oracle as orc

    out = str(tmp_path / "rank0.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    full = oracle_state(config0_ions(N_IONS))
    r = orc.run(config0_ensemble(), full, STEPS, integrator=0, collision=2, seed=123, snap_every=SNAP,
                ref_step=SNAP)
    np.testing.assert_allclose(got["moments"], r["moments"], rtol=1e-12, atol=1e-300)
    assert got["counts"].tolist() == [float(r["candidates"]), float(r["collisions"])]
    assert r["collisions"] > 0


class _FakeShard:
    """Stands for a rank's handle: its export writes its ions' rows, its
    set_peers records the list it is handed."""

    def __init__(self, rows: np.ndarray):
        self.rows = np.ascontiguousarray(rows, dtype=np.float64)
        self.peers = None

    def spacecharge_export(self, ptr: int) -> None:
        import ctypes
        ctypes.memmove(ptr, self.rows.ctypes.data, self.rows.nbytes)

    def set_spacecharge_peers(self, ptr: int, n: int, skip_begin: int = 0, skip_count: int = 0) -> None:
        import ctypes
        data = np.frombuffer(ctypes.string_at(ptr, n * 32), dtype=np.float64).reshape(n, 4).copy()
        self.peers = (data, skip_begin, skip_count)


def _sc_worker(rank: int, world: int, port: int, out_path: str) -> None:
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    from icarion_b200 import parallel

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n_total, n_max = 7, 4
        b, e = parallel.shard_range(n_total, rank, world)
        rows = np.array([[i, 10 * i, 100 * i, 1.0 + i] for i in range(b, e)], dtype=np.float64)
        fake = _FakeShard(rows)
        ex = parallel.SpaceChargeExchange(fake, e - b, n_max)
        ex.step()
        data, skip_b, skip_n = fake.peers
        np.savez(out_path + f".{rank}.npz", data=data, skip=np.array([skip_b, skip_n]))
    finally:
        dist.destroy_process_group()


def test_space_charge_exchange_gives_every_rank_all_ions(tmp_path):
    """Two gloo ranks with 4 and 3 of 7 ions (row blocks of 4): each gets
    the whole list, its own block as the skip range, and q = 0 in the
    padding rows."""
    out = str(tmp_path / "sc")
    mp.start_processes(_sc_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    for rank in (0, 1):
        got = np.load(out + f".{rank}.npz")
        data, skip = got["data"], got["skip"]
        assert data.shape == (8, 4)
        assert skip.tolist() == [4 * rank, 4]
        ions = np.concatenate([data[0:4], data[4:7]])
        np.testing.assert_array_equal(ions[:, 0], np.arange(7, dtype=np.float64))
        np.testing.assert_array_equal(ions[:, 3], 1.0 + np.arange(7, dtype=np.float64))
        assert data[7, 3] == 0.0
