"""Batched E/N sweep: many IMS ensembles advanced by one launch sequence.

The reference runs one domain per simulation; a sweep over E/N (its
``validation/configs/performance`` runs, one JSON per field) becomes one
handle here whose ensembles differ in field, species and dt and are
advanced by the same fused kernel (per-ensemble constants in the kernel's
parameter block, ions grouped by ensemble).

Default sweep: 64 ensembles, E/N log-spaced over 2-100 Td at 1000 Pa and
300 K in N2; species (100 Da, 100 A^2), (500 Da, 250 A^2), (2000 Da,
600 A^2) taken round-robin; ion counts exp(U(ln 1k, ln 256k)) from a fixed
seed; dt = 0.1 / nu_max of the ensemble, where

    nu_max = n sigma (<g> + 6 sigma_g)

is an upper estimate of the hard-sphere collision frequency at that field:
the relative speed g is Maxwellian in the reduced mass mu at Wannier's
effective temperature T_eff = T + M v_d^2 / (3 k) (M = gas mass), and the
drift speed v_d = K E comes from the first-order Chapman-Enskog hard-sphere
mobility K = (3 q / (16 n)) sqrt(2 pi / (mu k T_eff)) / sigma, iterated to
a fixed point (Mason & McDaniel, Transport Properties of Ions in Gases,
1988, ch. 5-6).  Everything else follows the single-ensemble IMS setup
(cylinder origin z = -1 cm, length 10 cm, radius 5 cm; Gaussian cloud of
0.5 mm at the origin; Maxwell-Boltzmann velocities at 300 K; detector plane
z = 2 mm).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import config as cfg
from .sim import IonState, generate_ions

SPECIES = ((100.0, 100.0), (500.0, 250.0), (2000.0, 600.0))   # (mass Da, HSS cross-section A^2)


def hard_sphere_drift(en_td: float, mass_kg: float, sigma_m2: float, gas_mass_kg: float, temperature_k: float,
                      pressure_pa: float, charge_c: float = cfg.ELEM_CHARGE_C, iters: int = 60) -> tuple[float, float]:
    """(v_d, T_eff): first-order hard-sphere mobility at Wannier's T_eff."""
    k = cfg.BOLTZMANN_CONSTANT
    n = cfg.gas_density(pressure_pa, temperature_k)
    e_field = en_td * 1e-21 * n
    mu = mass_kg * gas_mass_kg / (mass_kg + gas_mass_kg)
    t_eff, v_d = temperature_k, 0.0
    for _ in range(iters):
        mob = (3.0 * charge_c / (16.0 * n)) * math.sqrt(2.0 * math.pi / (mu * k * t_eff)) / sigma_m2
        v_d = mob * e_field
        t_eff = temperature_k + gas_mass_kg * v_d * v_d / (3.0 * k)
    return v_d, t_eff


def collision_frequency_max(en_td: float, mass_kg: float, sigma_m2: float, gas_mass_kg: float,
                            temperature_k: float, pressure_pa: float) -> float:
    """nu_max = n sigma (<g> + 6 sigma_g) with g Maxwellian at T_eff."""
    k = cfg.BOLTZMANN_CONSTANT
    n = cfg.gas_density(pressure_pa, temperature_k)
    mu = mass_kg * gas_mass_kg / (mass_kg + gas_mass_kg)
    _, t_eff = hard_sphere_drift(en_td, mass_kg, sigma_m2, gas_mass_kg, temperature_k, pressure_pa)
    g_mean = math.sqrt(8.0 * k * t_eff / (math.pi * mu))
    g_sd = math.sqrt(max(3.0 * k * t_eff / mu - g_mean * g_mean, 0.0))
    return n * sigma_m2 * (g_mean + 6.0 * g_sd)


@dataclass
class Sweep:
    ensembles: list           # ensemble parameter dicts (config.ensemble_params)
    en_td: np.ndarray         # E/N of each ensemble [Td]
    species: np.ndarray       # species index of each ensemble (into SPECIES)
    counts: np.ndarray        # ions per ensemble
    offsets: np.ndarray       # ion index ranges: ensemble e = [offsets[e], offsets[e+1])
    ions: IonState            # initial state, grouped by ensemble

    @property
    def n_ions(self) -> int:
        return int(self.offsets[-1])


def en_sweep(n_ensembles: int = 64, en_min_td: float = 2.0, en_max_td: float = 100.0,
             count_min: int = 1000, count_max: int = 256 * 1024, count_seed: int = 123, ion_seed: int = 123,
             pressure_pa: float = 1000.0, temperature_k: float = 300.0, gas: str = "N2",
             species: tuple = SPECIES, counts: np.ndarray | None = None, dt_fraction: float = 0.1) -> Sweep:
    """Build the sweep: ensemble parameters, counts and the initial ions
    (all species generated in ensemble order from one std::mt19937(ion_seed)
    stream, the reference IonLoader's semantics)."""
    en = np.geomspace(en_min_td, en_max_td, n_ensembles)
    sp = np.arange(n_ensembles) % len(species)
    if counts is None:
        rng = np.random.default_rng(count_seed)
        counts = np.exp(rng.uniform(math.log(count_min), math.log(count_max), n_ensembles)).astype(np.int64)
    counts = np.asarray(counts, dtype=np.int64)
    gas_mass = cfg.GAS_MASS_KG[gas]
    ensembles, specs = [], []
    for e in range(n_ensembles):
        m_da, ccs_a2 = species[sp[e]]
        mass = m_da * cfg.AMU_TO_KG
        sigma = ccs_a2 * cfg.ANGSTROM2_TO_M2
        nu = collision_frequency_max(float(en[e]), mass, sigma, gas_mass, temperature_k, pressure_pa)
        domain = {"instrument": "IMS",
                  "geometry": {"origin_m": [0.0, 0.0, -0.01], "length_m": 0.1, "radius_m": 0.05},
                  "env": {"temperature_K": temperature_k, "pressure_Pa": pressure_pa, "gas_species": gas},
                  "fields": {"DC": {"EN_Td": float(en[e])}}}
        ensembles.append(cfg.ensemble_params(domain, sigma, dt_fraction / nu, detector_z_m=2.0e-3))
        specs.append(cfg.species_spec(int(counts[e]), mass, cfg.ELEM_CHARGE_C,
                                      {"type": "gaussian", "center": [0, 0, 0], "std": [5e-4] * 3},
                                      {"type": "thermal", "temperature_K": temperature_k}))
    ions = generate_ions(ion_seed, specs)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    return Sweep(ensembles=ensembles, en_td=en, species=sp, counts=counts, offsets=offsets, ions=ions)


def subset(st: IonState, lo: int, hi: int) -> IonState:
    """Ions [lo, hi) of a state (for running one ensemble alone)."""
    return IonState(**{k: (None if v is None else np.ascontiguousarray(v[lo:hi])) for k, v in st.__dict__.items()})
