"""Device runs written through the snapshot writer (Simulation.run with a
TrajectoryWriter): the reference's /trajectory datasets (time, positions,
velocities, species ids) at every write_interval hold exactly the state the
library downloads at that step, and the times are the device clock's."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import config0_ensemble, config0_ions
from icarion_b200 import _capi as capi
from icarion_b200 import snapshots
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_written_snapshots_equal_the_downloaded_state(tmp_path, precision):
    n, interval, steps = 2000, 250, 1000
    e = config0_ensemble()
    st0 = config0_ions(n)
    species = np.zeros(n, dtype=np.uint32)
    species[1::2] = 1
    w = snapshots.TrajectoryWriter(tmp_path / "traj.npz", ["ion_a", "ion_b"], species)
    with Simulation([e], precision=precision, collision=capi.COLLISION_HSS, rng_seed=5) as sim:
        sim.upload(st0)
        steps_idx, mom, _ = sim.run(steps, interval, writer=w)
    d = snapshots.read(w.close())
    # the same run stepped by hand, downloaded at every interval
    want_pos, want_vel = [], []
    with Simulation([e], precision=precision, collision=capi.COLLISION_HSS, rng_seed=5) as sim:
        sim.upload(st0)
        for _ in range(steps // interval):
            sim.advance(interval)
            o = sim.download()
            want_pos.append(np.stack([o.x, o.y, o.z], axis=1))
            want_vel.append(np.stack([o.vx, o.vy, o.vz], axis=1))
    assert d["trajectory/positions"].shape == (steps // interval, n, 3)
    np.testing.assert_array_equal(d["trajectory/positions"], np.stack(want_pos))
    np.testing.assert_array_equal(d["trajectory/velocities"], np.stack(want_vel))
    np.testing.assert_allclose(d["trajectory/time"], steps_idx * e["dt_s"], rtol=1e-12)
    assert list(d["trajectory/species_ids"]) == ["ion_a", "ion_b"]
    np.testing.assert_array_equal(d["trajectory/species_id_indices"][-1], species)
    assert list(steps_idx) == [250, 500, 750, 1000] and mom.shape == (4, 1, capi.N_MOMENTS)
