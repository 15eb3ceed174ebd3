"""Space charge with the ions sharded over ranks (icb_spacecharge_export /
icb_spacecharge_set_peers), on one GPU: two handles stand for two ranks,
each holding half of the FT-ICR golden cloud (1,024 ions), and exchange
their ions through a device buffer before every step, as
`parallel.SpaceChargeExchange` does with an NCCL all-gather.

Against one handle with all the ions:
  * the field of every ion agrees to 1e-12 of the RMS field with the FP64
    solver, 1e-5 with the single-precision one (only the order of the
    deposit and pair sums differs: the sharded solve sorts own ions before
    peers within a cell);
  * after 200 steps with space charge the positions agree to 1e-9 (FP64
    solver) or 1e-4 (single precision) of the displacement's RMS size;
  * a rank's export gives its active ions' positions and charges and q = 0
    for the others, and a solve whose only peers are its own ions (skipped)
    equals the solve without peers bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from icarion_b200 import _capi as capi
from icarion_b200 import fticr
from icarion_b200.sim import IonState, Simulation, device_count

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def _cloud(z, sl=slice(None)):
    keys = ("x", "y", "z", "vx", "vy", "vz", "mass", "charge")
    arr = {k: np.ascontiguousarray(z["in_" + k][sl]) for k in keys}
    n = arr["x"].shape[0]
    return IonState(**arr, active=np.ones(n, dtype=np.uint8), t_death=None, t_arrival=None)


def _sim(cell, st, stream_ptr, solver_fp32=False):
    sim = Simulation([cell.ensemble], precision=capi.PREC_FP64, collision=capi.COLLISION_NONE, rng_seed=1)
    sim.set_stream(stream_ptr)
    sim.upload(st)
    fticr.configure(sim, cell, solver_fp32=solver_fp32)
    return sim


@pytest.mark.parametrize("solver_fp32,field_tol,pos_tol", [(False, 1e-12, 1e-9), (True, 1e-5, 1e-4)])
def test_sharded_solve_equals_the_whole_solve(golden, solver_fp32, field_tol, pos_tol):
    """FP64 solver: fields to 1e-12 of the RMS field, positions to 1e-9 of
    the space-charge displacement.  Single-precision solver (the 128^3
    mesh's fused x pass, float particle-particle sums in another order):
    1e-5 and 1e-4."""
    import torch
    z = golden("fticr_sc_direct.npz")
    n = int(z["n_ions"])
    cell = fticr.fticr_cell(n_ions=n, cloud_sigma_m=float(z["sigma_m"]))
    stream = torch.cuda.current_stream().cuda_stream
    half = n // 2
    whole = _sim(cell, _cloud(z), stream, solver_fp32)
    ranks = [_sim(cell, _cloud(z, slice(0, half)), stream, solver_fp32),
             _sim(cell, _cloud(z, slice(half, n)), stream, solver_fp32)]
    buf = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    blocks = [(0, half), (half, n - half)]

    def exchange():
        for sim, (b, m) in zip(ranks, blocks):
            sim.spacecharge_export(buf[b:b + m].data_ptr())
        for sim, (b, m) in zip(ranks, blocks):
            sim.set_spacecharge_peers(buf.data_ptr(), n, b, m)

    try:
        exchange()
        torch.cuda.synchronize()
        rows = buf.cpu().numpy()
        assert np.array_equal(rows[:, 0], z["in_x"]) and np.array_equal(rows[:, 3], z["in_charge"])
        f_whole = whole.space_charge_field()
        f_split = np.concatenate([r.space_charge_field() for r in ranks], axis=1)
        rms = float(np.sqrt(np.mean(np.sum(f_whole ** 2, axis=0))))
        err = float(np.max(np.abs(f_split - f_whole)))
        assert rms > 0 and err <= field_tol * rms, (err, rms)

        x0 = np.stack([z["in_" + k] for k in ("x", "y", "z")])
        for _ in range(200):
            exchange()
            for sim in ranks:
                sim.advance(1)
        whole.advance(200)
        out_w = whole.download()
        outs = [r.download() for r in ranks]
        pw = np.stack([out_w.x, out_w.y, out_w.z])
        ps = np.concatenate([np.stack([o.x, o.y, o.z]) for o in outs], axis=1)
        disp = float(np.sqrt(np.mean(np.sum((pw - x0) ** 2, axis=0))))
        print("sharded vs whole: field", err / rms, "positions", float(np.max(np.abs(ps - pw))) / disp)
        assert float(np.max(np.abs(ps - pw))) <= pos_tol * disp
    finally:
        for s in [whole] + ranks:
            s.close()


def test_export_marks_inactive_ions_and_own_skip_changes_nothing(golden):
    import torch
    z = golden("fticr_sc_direct.npz")
    n = int(z["n_ions"])
    cell = fticr.fticr_cell(n_ions=n, cloud_sigma_m=float(z["sigma_m"]))
    st = _cloud(z)
    st.active[::5] = 0
    stream = torch.cuda.current_stream().cuda_stream
    sim = _sim(cell, st, stream)
    try:
        buf = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
        f0 = sim.space_charge_field()
        sim.spacecharge_export(buf.data_ptr())
        torch.cuda.synchronize()
        rows = buf.cpu().numpy()
        act = st.active != 0
        assert np.array_equal(rows[act, 2], st.z[act]) and np.array_equal(rows[act, 3], st.charge[act])
        assert np.all(rows[~act, 3] == 0.0)
        sim.set_spacecharge_peers(buf.data_ptr(), n, 0, n)       # only itself, skipped
        f1 = sim.space_charge_field()
        assert np.array_equal(f0, f1)
        sim.set_spacecharge_peers(0, 0)
        assert np.array_equal(sim.space_charge_field(), f0)
    finally:
        sim.close()
