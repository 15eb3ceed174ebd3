"""The interaction-potential collision law pinned to the reference's own
runtime sampler (CPU).

Fixture ipm_ref_40Td.npz (tests/golden/make_ipm_golden.py): the reference's
InteractionPotentialCollisionHandler (compiled from its sources) with an
offline sample set built by the reference tool's per-cell rule from the
restated deflection quadrature, 65,536 ions of 300 Da in N2 at 40 Td, 30,000
steps.  The reference samples a momentum transfer of the nearer log-speed bin
(stochastically interpolated) from per-cell CDFs; this library deflects the
relative velocity by chi(E, b) at the collision's own energy.  The two are
the same collision law up to the sample set's speed binning, so the
observables must agree.

Tolerances: v_drift, K0, D_L, D_T within 4 combined standard errors (the
fixture's and the oracle run's, independent ions); collision fraction within
4 sqrt(2 / collisions) relative (counting noise of both runs).
"""
from __future__ import annotations

import math

import numpy as np

import oracle as orc
from helpers import assert_transport_close, ipm_reference_case, oracle_state

AMU = 1.66053906660e-27
EV = 1.602176634e-19


def test_restated_quadrature_matches_trajectory_integrator():
    """The oracle's CPU quadrature (used for the sample set and the CPU
    table) against the restated trajectory integrator of the reference
    tool: |d cos(chi)| <= 1e-3 on an (E, b) grid."""
    from icarion_b200 import ipm
    s = ipm.IpmSetup()
    c12, c6, c4 = s.coefficients()
    sigma = s.r_m_m * 2.0 ** (-1.0 / 6.0)
    mu = 300 * 28.0134 / 328.0134 * AMU
    E = np.repeat(np.array([10, 26, 50, 100, 300, 1000, 3000, 10000]) * 1e-3 * EV, 13)
    b = np.tile(np.arange(13) * 1e-10, 8)
    got = orc.ipm_cos_chi_quad(c12, c6, c4, sigma, E, b)
    want = np.array([orc.ipm_cos_chi_trajectory(c12, c6, c4, mu, e, bb) for e, bb in zip(E, b)])
    assert np.max(np.abs(got - want)) <= 1e-3


def test_oracle_table_collisions_match_reference_handler(golden):
    z = golden("ipm_ref_40Td.npz")
    setup, e, st0, fit = ipm_reference_case(z)
    c12, c6, c4 = setup.coefficients()
    tab = orc.ipm_table(c12, c6, c4, setup.r_m_m * 2.0 ** (-1.0 / 6.0), setup.n_E, setup.n_b, setup.table_E_min_J,
                        setup.E_max_J, setup.b_max_m)
    orc.set_ipm_table(tab.ravel(), setup.n_E, setup.n_b, *setup.table_scale())
    n, steps = int(z["n_ions"]), int(z["steps"])
    ost = oracle_state(st0)
    r = orc.run(e, ost, steps, integrator=0, collision=4, seed=int(z["seed"]), snap_every=int(z["snap_every"]),
                ref_step=int(z["ref_step"]), threads=8)
    ref, got = fit(z["moments"]), fit(r["moments"])
    assert_transport_close(got, ref)
    c_ref, c_got = float(z["collisions"]), float(r["collisions"])
    assert abs(c_got / c_ref - 1.0) <= 4.0 * math.sqrt(2.0 / c_ref), (c_got, c_ref)
    assert c_ref > 0.05 * n * steps
