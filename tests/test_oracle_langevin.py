"""Langevin capture collisions in the oracle (CPU): the event count matches
the constant per-ion rate nu = n pi |q| sqrt(alpha' / (4 pi eps0 mu))
(sigma_L(v) v of DampingForce.cpp:170-176), and collisions drive a cold
beam towards the gas temperature."""
from __future__ import annotations

import math

import numpy as np

import oracle as orc
from helpers import config0_ensemble, config0_ions, oracle_state
from icarion_b200 import config as cfg


def test_langevin_event_count_matches_rate():
    e = config0_ensemble()
    st = oracle_state(config0_ions(2000))
    steps = 2000
    r = orc.run(e, st, steps, integrator=0, collision=3, seed=9)
    m = 200 * cfg.AMU_TO_KG
    mu = m * e["gas_mass_kg"] / (m + e["gas_mass_kg"])
    lam = e["gas_density_m3"] * e["dt_s"] * math.pi * cfg.ELEM_CHARGE_C * math.sqrt(
        e["gas_polarizability_m3"] / (4 * math.pi * cfg.EPSILON_0 * mu))
    p = -math.expm1(-lam)
    want = 2000 * steps * p
    assert abs(r["collisions"] - want) < 4 * math.sqrt(want * (1 - p))
    assert r["candidates"] == r["collisions"]


def test_langevin_thermalises_a_cold_beam():
    e = config0_ensemble()
    e["axial_V"] = 0.0
    st = oracle_state(config0_ions(2000))
    st["vx"][:] = 0.0
    st["vy"][:] = 0.0
    st["vz"][:] = 2000.0                      # a fast, cold beam
    orc.run(e, st, 6000, integrator=0, collision=3, seed=10)
    m = 200 * cfg.AMU_TO_KG
    t_ion = m * np.var(np.concatenate([st["vx"], st["vy"], st["vz"] - st["vz"].mean()])) / cfg.BOLTZMANN_CONSTANT
    assert abs(np.mean(st["vz"])) < 200.0     # beam stopped (about 200 collisions per ion)
    assert 240.0 < t_ion < 360.0              # at the gas temperature (300 K) within sampling noise
