"""Collision sub-steps (CPU): with m sub-steps the reference engine repeats
the collision test m times per step with dt/m at the pushed position
(SimulationEngineCollisionRuntime.cpp:79-190), so an ion can collide more
than once per step.  The oracle's plain form (Philox words) against the
reference's own handler looped the same way (compiled harness), m = 4 at
4000 Pa (about 0.35 collisions per step): collisions per ion-step within
1.5 %, drift and mean energy within 4 combined standard errors; m = 1 keeps
the one-test form bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from helpers import CONFIG0_DOMAIN, config0_ions, domain_json, oracle_state
from icarion_b200 import config as cfg

DOMAIN = dict(CONFIG0_DOMAIN, P=4000)


def dense_ensemble():
    return cfg.ensemble_params(domain_json(DOMAIN), 150e-20, 5e-10)


def test_one_substep_is_the_plain_form():
    st0 = config0_ions(256)
    a, b = oracle_state(st0), oracle_state(st0)
    ra = orc.run(dense_ensemble(), a, 500, integrator=0, collision=6, seed=5)
    rb = orc.run(dense_ensemble(), b, 500, integrator=0, collision=6, seed=5, subcycles=1)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(a[k], b[k]), k
    assert ra["collisions"] == rb["collisions"]


@pytest.mark.skipif(not orc.HARNESS.exists(), reason="compiled reference harness not built")
def test_substeps_match_reference_handler():
    n, steps, m = 2048, 3000, 4
    st0 = config0_ions(n)
    ref_state = oracle_state(st0)
    ref_state["ccs"] = np.full(n, 150e-20)
    rst, rstats, _ = orc.harness_run(ref_state, steps, dict(DOMAIN, subcycles=m), integrator="boris",
                                     collision="hss", dt=5e-10, seed=11, threads=8)
    ost = oracle_state(st0)
    r = orc.run(dense_ensemble(), ost, steps, integrator=0, collision=6, seed=11, threads=8, subcycles=m)
    f_ref, f_me = rstats["collisions"] / (n * steps), r["collisions"] / (n * steps)
    assert f_ref > 0.3
    assert abs(f_me / f_ref - 1.0) < 0.015, (f_me, f_ref)
    one = orc.run(dense_ensemble(), oracle_state(st0), steps, integrator=0, collision=6, seed=11, threads=8)
    assert r["collisions"] > 1.05 * one["collisions"]      # more than one collision per step happens
    dz_ref, dz_me = rst["z"] - st0.z, ost["z"] - st0.z
    se = np.hypot(dz_ref.std(), dz_me.std()) / np.sqrt(n)
    assert abs(dz_me.mean() - dz_ref.mean()) <= 4 * se
    ke_ref = rst["vx"] ** 2 + rst["vy"] ** 2 + rst["vz"] ** 2
    ke_me = ost["vx"] ** 2 + ost["vy"] ** 2 + ost["vz"] ** 2
    se_ke = np.hypot(ke_ref.std(), ke_me.std()) / np.sqrt(n)
    assert abs(ke_me.mean() - ke_ref.mean()) <= 4 * se_ke
