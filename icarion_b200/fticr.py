"""FT-ICR cell with space charge: the ion cloud, the trap ensemble and the
mesh of its space-charge solve.

Default cell: 262,144 singly charged ions with m/z uniform over 500-1500 in
the reference's FTICR quadrupolar trap (AnalyticalFieldModel.cpp:174-186:
E = (V/d^2)(x, y, -2(z - L/2)), d^2 = L^2/8 + r^2/4, z global) with
radial_V = 1 V, a 5 cm long cylinder of 2.5 cm radius from z = 0 to z = L
(the field model centres the trap at global z = L/2, so the cylinder starts
at z = 0 as the reference's FT-ICR setups place it), B = 7 T along z, and
He at 1e-7 Pa and 300 K with Langevin capture collisions.  The cloud is a
Gaussian of 1 mm per axis centred 2 mm off the axis in the trap's mid-plane
(x = 2 mm, z = L/2) moving with the cyclotron velocity v_y = -omega_c * 2 mm
of each ion (the state after a coherent excitation to a 2 mm cyclotron
radius, omega_c = qB/m), plus Maxwell-Boltzmann velocities at 300 K.  Boris
push, dt = 1e-9 s.  Space charge: isolated P3M on a 128^3 mesh over a
14 mm cube around the trap centre (cyclotron orbits stay within about 6 mm
of the axis), CIC, particle-particle correction within 2 cells.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _capi as capi
from . import config as cfg
from .sim import IonState, generate_ions


@dataclass
class FticrCell:
    ensemble: dict
    ions: IonState
    sc_grid: tuple
    sc_box_min: tuple
    sc_box_max: tuple


def fticr_cell(n_ions: int = 262_144, seed: int = 123, mz_min: float = 500.0, mz_max: float = 1500.0,
               b_tesla: float = 7.0, radial_v: float = 1.0, cyclotron_radius_m: float = 2e-3,
               cloud_sigma_m: float = 1e-3, pressure_pa: float = 1e-7, temperature_k: float = 300.0,
               dt_s: float = 1e-9, mesh: int = 128, box_half_m: float = 7e-3) -> FticrCell:
    length, radius = 0.05, 0.025
    domain = {"instrument": "FTICR",
              "geometry": {"origin_m": [0.0, 0.0, 0.0], "length_m": length, "radius_m": radius},
              "env": {"temperature_K": temperature_k, "pressure_Pa": pressure_pa, "gas_species": "He"},
              "fields": {"DC": {"radial_V": radial_v},
                         "magnetic": {"enabled": True, "field_strength_T": [0.0, 0.0, b_tesla]}}}
    ens = cfg.ensemble_params(domain, 1e-20, dt_s)
    # positions and thermal velocities with the reference loader's semantics
    # (one species per call keeps the mt19937 stream order), then the m/z
    # draw and the coherent cyclotron velocity from a separate seeded stream
    spec = cfg.species_spec(n_ions, 1000.0 * cfg.AMU_TO_KG, cfg.ELEM_CHARGE_C,
                            {"type": "gaussian", "center": [cyclotron_radius_m, 0.0, length / 2],
                             "std": [cloud_sigma_m] * 3},
                            {"type": "thermal", "temperature_K": temperature_k})
    st = generate_ions(seed, [spec])
    rng = np.random.default_rng(seed)
    mz = rng.uniform(mz_min, mz_max, n_ions)
    mass = mz * cfg.AMU_TO_KG
    # thermal velocities were drawn for 1000 Da: rescale to each ion's mass
    scale = np.sqrt(1000.0 * cfg.AMU_TO_KG / mass)
    st.vx *= scale
    st.vy *= scale
    st.vz *= scale
    st.mass[:] = mass
    omega_c = cfg.ELEM_CHARGE_C * b_tesla / mass
    st.vy -= omega_c * cyclotron_radius_m
    h, zc = box_half_m, length / 2
    return FticrCell(ensemble=ens, ions=st, sc_grid=(mesh, mesh, mesh), sc_box_min=(-h, -h, zc - h),
                     sc_box_max=(h, h, zc + h))


def configure(sim, cell: FticrCell, mode: int = capi.SC_P3M_ISOLATED, solver_fp32: bool = False) -> None:
    sim.configure_space_charge(mode, cell.sc_grid, cell.sc_box_min, cell.sc_box_max, solver_fp32=solver_fp32)
