"""Snapshot writer layout (CPU): the reference's /trajectory datasets."""
from __future__ import annotations

import numpy as np

from icarion_b200 import snapshots
from icarion_b200.sim import IonState


def test_writer_layout_round_trip(tmp_path):
    n = 5
    w = snapshots.TrajectoryWriter(tmp_path / "traj.npz", ["A", "B"], np.array([0, 1, 1, 0, 1]))
    for k in range(3):
        st = IonState.empty(n)
        st.x[:] = k
        st.vz[:] = -k
        w.append(k * 1e-6, st)
    d = snapshots.read(w.close())
    assert d["trajectory/positions"].shape == (3, n, 3)
    assert d["trajectory/velocities"].shape == (3, n, 3)
    np.testing.assert_array_equal(d["trajectory/time"], [0.0, 1e-6, 2e-6])
    assert np.all(d["trajectory/positions"][2, :, 0] == 2.0)
    assert np.all(d["trajectory/velocities"][1, :, 2] == -1.0)
    assert list(d["trajectory/species_ids"]) == ["A", "B"]
    assert d["trajectory/species_id_indices"].shape == (3, n)
