"""Trajectory snapshots in the reference's output layout.

The reference's HDF5 writer keeps one group /trajectory with, per snapshot,
time[F], positions[F, N, 3], velocities[F, N, 3] and the per-ion species
index species_id_indices[F, N], plus the species names species_ids[S]
(hdf5Writer.cpp:147, 296-298, 652-656).  HDF5 is not available here, so the
writer stores the same datasets under the same paths ("trajectory/time",
...) in an uncompressed .npz; reading one back gives the arrays the
reference's analysis scripts take from the HDF5 file.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .sim import IonState


class TrajectoryWriter:
    def __init__(self, path: str | Path, species_ids: list[str], species_index: np.ndarray):
        self.path = Path(path)
        self.species_ids = list(species_ids)
        self.species_index = np.asarray(species_index, dtype=np.uint32)
        self.times: list[float] = []
        self.pos: list[np.ndarray] = []
        self.vel: list[np.ndarray] = []

    def append(self, t: float, st: IonState) -> None:
        """One snapshot (hdf5Writer::write_timestep, :296-298)."""
        self.times.append(float(t))
        self.pos.append(np.stack([st.x, st.y, st.z], axis=1).astype(np.float64))
        self.vel.append(np.stack([st.vx, st.vy, st.vz], axis=1).astype(np.float64))

    def close(self) -> Path:
        f = len(self.times)
        n = self.species_index.size
        data = {
            "trajectory/time": np.asarray(self.times, dtype=np.float64),
            "trajectory/positions": np.stack(self.pos) if f else np.zeros((0, n, 3)),
            "trajectory/velocities": np.stack(self.vel) if f else np.zeros((0, n, 3)),
            "trajectory/species_id_indices": np.tile(self.species_index, (f, 1)),
            "trajectory/species_ids": np.asarray(self.species_ids),
        }
        with open(self.path, "wb") as fh:
            np.savez(fh, **data)
        return self.path


def read(path: str | Path) -> dict:
    with np.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}
