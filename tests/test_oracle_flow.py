"""Gas-flow profiles (CPU): the oracle's null-collision HSS with the flow
evaluated at each colliding ion (EnvironmentConfig::gas_velocity_at,
EnvironmentConfig.h:96-128, as SimulationEngineCollisionRuntime.cpp:124-131
applies it) against the reference's own handler and flow code (compiled
harness) on the same cloud in a 1.2 mm cylinder: collision fraction within
1.5 %, mean axial displacement of the surviving ions within 4 combined
standard errors overall and in three radial bins (the parabolic profile
drifts the axis ions ~50 % further than those near the wall)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from helpers import CONFIG0_DOMAIN, config0_ions, domain_json, oracle_state
from icarion_b200 import _capi as capi
from icarion_b200 import config as cfg

RADIUS = 1.2e-3
CASES = {
    "axial_parabolic": ({"axial_flow_max_velocity_m_s": 100.0}, {"axial_flow_max_velocity": 100.0}),
    "axial_uniform": ({"axial_flow_velocity_m_s": 60.0}, {"axial_flow_velocity": 60.0}),
}


def flow_ensemble(model: str, env_kw: dict) -> dict:
    dom = domain_json(CONFIG0_DOMAIN)
    dom["geometry"]["radius_m"] = RADIUS
    dom["env"]["flow_model"] = model
    dom["env"].update(env_kw)
    return cfg.ensemble_params(dom, 150e-20, 5e-10)


def test_flow_model_names_follow_the_loader():
    assert cfg.flow_model("Legacy") == capi.FLOW_CONSTANT
    assert cfg.flow_model("axial_const") == capi.FLOW_AXIAL_UNIFORM
    assert cfg.flow_model("Poiseuille") == capi.FLOW_AXIAL_PARABOLIC
    with pytest.raises(ValueError):
        cfg.flow_model("swirl")
    e = flow_ensemble("parabolic", {"axial_flow_max_velocity_m_s": 3.0})
    assert e["flow_model"] == capi.FLOW_AXIAL_PARABOLIC and e["axial_flow_max_velocity_m_s"] == 3.0


@pytest.mark.skipif(not orc.HARNESS.exists(), reason="compiled reference harness not built")
@pytest.mark.parametrize("model", sorted(CASES))
def test_flow_oracle_matches_reference(model):
    env_kw, harness_kw = CASES[model]
    n, steps = 4096, 6000
    st0 = config0_ions(n)
    ref_state = oracle_state(st0)
    ref_state["ccs"] = np.full(n, 150e-20)
    rst, rstats, _ = orc.harness_run(ref_state, steps, dict(CONFIG0_DOMAIN, radius=RADIUS, flow_model=model,
                                                            **harness_kw),
                                     integrator="boris", collision="hss", dt=5e-10, seed=11, threads=8)
    ost = oracle_state(st0)
    r = orc.run(flow_ensemble(model, env_kw), ost, steps, integrator=0, collision=2, seed=11, threads=8)
    f_ref, f_me = rstats["collisions"] / (n * steps), r["collisions"] / (n * steps)
    assert abs(f_me / f_ref - 1.0) < 0.015, (f_me, f_ref)
    rr = np.hypot(st0.x, st0.y)
    for lo, hi in ((0.0, 1.0), (0.0, 4e-4), (4e-4, 8e-4), (8e-4, RADIUS)):
        m_ref = (rst["active"] != 0) & (rr >= lo) & (rr < hi)
        m_me = (ost["active"] != 0) & (rr >= lo) & (rr < hi)
        assert m_ref.sum() > 500 and abs(int(m_ref.sum()) - int(m_me.sum())) <= 0.01 * m_ref.sum()
        dz_ref, dz_me = (rst["z"] - st0.z)[m_ref], (ost["z"] - st0.z)[m_me]
        se = np.hypot(dz_ref.std() / np.sqrt(dz_ref.size), dz_me.std() / np.sqrt(dz_me.size))
        assert abs(dz_me.mean() - dz_ref.mean()) <= 4 * se, (lo, hi, dz_me.mean(), dz_ref.mean(), se)
