"""Host-side E/N sweep builder: ensemble layout, counts, dt rule."""
from __future__ import annotations

import math

import numpy as np

from icarion_b200 import config as cfg
from icarion_b200 import sweep


def test_default_sweep_layout():
    sw = sweep.en_sweep()
    assert len(sw.ensembles) == 64
    np.testing.assert_allclose(sw.en_td[[0, -1]], [2.0, 100.0])
    np.testing.assert_allclose(np.diff(np.log(sw.en_td)), math.log(50.0) / 63)
    assert list(sw.species[:6]) == [0, 1, 2, 0, 1, 2]
    assert sw.counts.min() >= 1000 and sw.counts.max() <= 256 * 1024
    assert sw.offsets[0] == 0 and sw.offsets[-1] == sw.counts.sum() == sw.ions.n
    assert 2_000_000 < sw.n_ions < 4_500_000
    for e in (0, 1, 2):
        lo, hi = int(sw.offsets[e]), int(sw.offsets[e + 1])
        m_da = sweep.SPECIES[sw.species[e]][0]
        assert np.all(sw.ions.mass[lo:hi] == m_da * cfg.AMU_TO_KG)
    # E/N -> axial voltage over the 10 cm cylinder (DomainConfigLoader arithmetic)
    n = cfg.gas_density(1000.0, 300.0)
    assert sw.ensembles[-1]["axial_V"] == 100.0 * 1e-21 * n * 0.1


def test_dt_rule_low_field_limit():
    """At vanishing field T_eff -> T and nu_max -> n sigma (<g> + 6 sigma_g)
    of a Maxwellian relative speed at the gas temperature."""
    k, T, P = cfg.BOLTZMANN_CONSTANT, 300.0, 1000.0
    m, M, sig = 500 * cfg.AMU_TO_KG, cfg.GAS_MASS_KG["N2"], 250e-20
    mu = m * M / (m + M)
    g = math.sqrt(8 * k * T / (math.pi * mu))
    sg = math.sqrt(3 * k * T / mu - g * g)
    want = cfg.gas_density(P, T) * sig * (g + 6 * sg)
    got = sweep.collision_frequency_max(1e-6, m, sig, M, T, P)
    assert abs(got / want - 1) < 1e-9
    # low-field hard-sphere mobility (3q/16n) sqrt(2 pi / (mu k T)) / sigma
    v_d, t_eff = sweep.hard_sphere_drift(1.0, m, sig, M, T, P)
    n = cfg.gas_density(P, T)
    k_mob = (3 * cfg.ELEM_CHARGE_C / (16 * n)) * math.sqrt(2 * math.pi / (mu * k * T)) / sig
    assert abs(v_d / (k_mob * 1e-21 * n) - 1) < 1e-3 and t_eff > T


def test_dt_shrinks_with_field_and_cross_section():
    sw = sweep.en_sweep(n_ensembles=6, counts=np.full(6, 10))
    dts = np.array([e["dt_s"] for e in sw.ensembles])
    assert np.all(dts > 0)
    # same species (index 0) at higher field -> hotter ions -> shorter dt
    assert dts[3] < dts[0]
