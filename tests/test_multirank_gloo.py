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
