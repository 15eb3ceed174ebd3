"""HSS gas mixtures (CPU): the oracle's exact null-collision restatement of
the reference's mixture law (HSSCollisionHandler.cpp:105-249) against the
reference's own handler (compiled harness) on the same cloud, with two and
five components: collision fraction within 1.5 %, drift and mean energy
within 4 combined standard errors."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from helpers import CONFIG0_DOMAIN, config0_ions, domain_json, oracle_state
from icarion_b200 import config as cfg

MIX = [("N2", 0.79, 150e-20), ("He", 0.21, 60e-20)]
# five components: the kernel takes up to eight
MIX5 = [("N2", 0.55, 150e-20), ("He", 0.15, 60e-20), ("Ar", 0.12, 130e-20), ("O2", 0.10, 140e-20),
        ("CO2", 0.08, 190e-20)]


def _mix_ensemble(mix=MIX):
    dom = domain_json(CONFIG0_DOMAIN)
    dom["env"]["gas_mixture"] = [{"species": s, "mole_fraction": f, "cross_section_m2": c} for s, f, c in mix]
    return cfg.ensemble_params(dom, 150e-20, 5e-10)


def test_mixture_constants_follow_the_loader():
    e = _mix_ensemble()
    n = cfg.gas_density(1000.0, 300.0)
    assert e["n_gas"] == 2
    np.testing.assert_allclose(e["gas_mix_density_m3"][:2], [0.79 * n, 0.21 * n], rtol=1e-15)
    assert e["gas_mix_mass_kg"][1] == cfg.GAS_MASS_KG["He"]
    assert e["gas_mix_sigma_m2"][:2] == [150e-20, 60e-20]


def test_components_outside_collisions_are_left_out():
    """participates_in_collisions = false drops a component from the
    collision law; its mole fraction still dilutes the others
    (EnvironmentConfig.h:155-175, HSSCollisionHandler.cpp:127-133)."""
    dom = domain_json(CONFIG0_DOMAIN)
    n = cfg.gas_density(1000.0, 300.0)
    dom["env"]["gas_mixture"] = [{"species": "N2", "mole_fraction": 0.5, "cross_section_m2": 150e-20},
                                 {"species": "He", "mole_fraction": 0.25, "cross_section_m2": 60e-20},
                                 {"species": "Ar", "mole_fraction": 0.25, "participates_in_collisions": False}]
    e = cfg.ensemble_params(dom, 150e-20, 5e-10)
    assert e["n_gas"] == 2
    np.testing.assert_allclose(e["gas_mix_density_m3"][:2], [0.5 * n, 0.25 * n], rtol=1e-15)
    dom["env"]["gas_mixture"][1]["participates_in_collisions"] = False
    e = cfg.ensemble_params(dom, 150e-20, 5e-10)
    assert e["n_gas"] == 0 and e["gas_density_m3"] == 0.5 * n and e["gas_mass_kg"] == cfg.GAS_MASS_KG["N2"]
    assert e["sigma_m2"] == 150e-20


def test_eight_components_accepted_nine_rejected():
    gases = ["N2", "He", "Ar", "O2", "CO2", "Ne", "H2O", "N2", "He"]
    dom = domain_json(CONFIG0_DOMAIN)
    dom["env"]["gas_mixture"] = [{"species": g, "mole_fraction": 1.0} for g in gases[:8]]
    assert cfg.ensemble_params(dom, 150e-20, 5e-10)["n_gas"] == 8
    dom["env"]["gas_mixture"] = [{"species": g, "mole_fraction": 1.0} for g in gases]
    with pytest.raises(ValueError):
        cfg.ensemble_params(dom, 150e-20, 5e-10)


@pytest.mark.skipif(not orc.HARNESS.exists(), reason="compiled reference harness not built")
@pytest.mark.parametrize("mix_def", [MIX, MIX5], ids=["2 gases", "5 gases"])
def test_mixture_oracle_matches_reference_handler(mix_def):
    n, steps = 2048, 6000
    st0 = config0_ions(n)
    ref_state = oracle_state(st0)
    ref_state["ccs"] = np.full(n, 150e-20)
    mix = ",".join(f"{s}:{f}:{c!r}" for s, f, c in mix_def)
    rst, rstats, _ = orc.harness_run(ref_state, steps, dict(CONFIG0_DOMAIN, mix=mix), integrator="boris",
                                     collision="hss", dt=5e-10, seed=11, threads=8)
    ost = oracle_state(st0)
    r = orc.run(_mix_ensemble(mix_def), ost, steps, integrator=0, collision=5, seed=11, threads=8)
    f_ref = rstats["collisions"] / (n * steps)
    f_me = r["collisions"] / (n * steps)
    assert abs(f_me / f_ref - 1.0) < 0.015, (f_me, f_ref)
    dz_ref, dz_me = rst["z"] - st0.z, ost["z"] - st0.z
    se = np.hypot(dz_ref.std(), dz_me.std()) / np.sqrt(n)
    assert abs(dz_me.mean() - dz_ref.mean()) <= 4 * se
    ke_ref = (rst["vx"] ** 2 + rst["vy"] ** 2 + rst["vz"] ** 2)
    ke_me = (ost["vx"] ** 2 + ost["vy"] ** 2 + ost["vz"] ** 2)
    se_ke = np.hypot(ke_ref.std(), ke_me.std()) / np.sqrt(n)
    assert abs(ke_me.mean() - ke_ref.mean()) <= 4 * se_ke
