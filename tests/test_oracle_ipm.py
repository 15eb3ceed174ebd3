"""Interaction-potential oracle pins (CPU).

* the numpy backpropagation of the deflection network against central
  finite differences (FP64);
* the restated reference trajectory integrator (interaction_potential_
  precompute.cpp:1672-1835; the tool itself needs HDF5 and jsoncpp and is
  not built here) against an independent adaptive quadrature of the
  classical deflection integral (scipy);
* the oracle's table collisions: event count at the rate n g pi b_max^2.
"""
from __future__ import annotations

import math

import numpy as np
import pytest
from scipy import integrate, optimize

import mlp as omlp
import oracle as orc
from helpers import config0_ensemble, config0_ions, oracle_state
from icarion_b200 import config as cfg
from icarion_b200.ipm import IpmSetup

EV = 1.602176634e-19
AMU = 1.66053906660e-27


def test_mlp_backprop_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, omlp.N_PARAMS)
    x = rng.uniform(-1, 1, (64, 2))
    y = rng.uniform(-1, 1, 64)
    _, g = omlp.loss_and_grad(p, x, y)
    idx = np.concatenate([rng.choice(128, 8, replace=False), 128 + rng.choice(64, 4, replace=False),
                          192 + rng.choice(4096, 16, replace=False), 4288 + rng.choice(64, 4, replace=False),
                          4352 + rng.choice(64, 4, replace=False), [4416]])
    for k in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (omlp.loss_and_grad(pp, x, y)[0] - omlp.loss_and_grad(pm, x, y)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-7 + 1e-5 * abs(g[k]), (k, fd, g[k])


def _quad_cos_chi(c12, c6, c4, E, b):
    """Independent evaluation: outermost turning point by root search on a
    fine grid, then adaptive quadrature of the deflection integral in the
    variable r = r0 / u with the 1/sqrt singularity removed by u = 1 - s^2."""
    def F(r):
        return 1.0 - b * b / (r * r) - (c12 / r ** 12 - c6 / r ** 6 - c4 / r ** 4) / E
    rs = np.geomspace(1e-11, 1e-8, 20000)[::-1]
    vals = np.array([F(r) for r in rs])
    k = int(np.argmax(vals <= 0.0))
    r0 = optimize.brentq(F, rs[k], rs[k - 1], xtol=1e-25, rtol=1e-15)
    I, _ = integrate.quad(lambda s: 2.0 * s / math.sqrt(max(F(r0 / (1.0 - s * s)), 1e-300)), 0.0, 1.0,
                          limit=400, epsabs=1e-11, epsrel=1e-11)
    return math.cos(math.pi - 2.0 * (b / r0) * I)


@pytest.mark.parametrize("E_meV", [10, 50, 300, 3000])
def test_trajectory_integrator_matches_quadrature(E_meV):
    s = IpmSetup()
    c12, c6, c4 = s.coefficients()
    mu = 300 * 28.0134 / 328.0134 * AMU
    E = E_meV * 1e-3 * EV
    for b_A in (0.0, 1.5, 3.0, 5.0, 8.0, 11.0):
        b = b_A * 1e-10
        t = orc.ipm_cos_chi_trajectory(c12, c6, c4, mu, E, b)
        q = _quad_cos_chi(c12, c6, c4, E, b)
        assert abs(t - q) < 1e-3, (E_meV, b_A, t, q)


def test_oracle_table_collision_rate():
    """With a table of cos(chi) = 1 (no deflection) the event count is the
    null-collision rate n g pi b_max^2 summed over steps (Poisson bound)."""
    s = IpmSetup(n_E=4, n_b=4)
    orc.set_ipm_table(np.ones(16, dtype=np.float32), 4, 4, math.log(s.E_min_J),
                      3 / (math.log(s.E_max_J) - math.log(s.E_min_J)))
    e = config0_ensemble()
    e["ipm_bmax_m"] = s.b_max_m
    e["axial_V"] = 0.0
    st = oracle_state(config0_ions(1000))
    steps = 1000
    r = orc.run(e, st, steps, integrator=0, collision=4, seed=5)
    # per-step probability 1 - exp(-n pi b_max^2 g dt), g the relative speed
    # of a thermal 200 Da ion and N2 at 300 K (Maxwellian in the reduced mass)
    mu = 200 * 28.0134 / 228.0134 * AMU
    g = np.linalg.norm(np.random.default_rng(1).normal(0.0, math.sqrt(cfg.BOLTZMANN_CONSTANT * 300 / mu),
                                                       (400000, 3)), axis=1)
    a = e["gas_density_m3"] * math.pi * s.b_max_m ** 2 * e["dt_s"]
    want = 1000 * steps * float(np.mean(-np.expm1(-a * g)))
    assert abs(r["collisions"] - want) < 5 * math.sqrt(want) + 0.01 * want
    assert np.allclose(np.hypot(np.hypot(st["vx"], st["vy"]), st["vz"]).mean(),
                       np.hypot(np.hypot(config0_ions(1000).vx, config0_ions(1000).vy),
                                config0_ions(1000).vz).mean(), rtol=0.05)
