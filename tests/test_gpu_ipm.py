"""Interaction-potential collisions and the learned deflection on the device.

Tolerances (stated per test):
  * device quadrature vs the restated reference trajectory integrator:
    |d cos(chi)| <= 1e-3 on an (E, b) grid (measured <= 3.3e-4);
  * the handle's table equals the quadrature at its nodes to float rounding;
  * FP64 table collisions vs the oracle with the same Philox streams:
    >= 99 % of ions to 1e-9 after 2000 steps, collision counts within 1 %;
  * network gradients (FP32 device) vs numpy FP64 backpropagation: relative
    norm error <= 1e-4; forward FP32 <= 1e-5 absolute; the BF16 tensor-core
    forward within 2e-2 of FP32 (BF16 weights and activations);
  * training lowers the loss tenfold;
  * learned vs table deflection: mean drift within 3 % at 40 Td;
  * device table collisions (FP64 and mixed) against the reference's own
    InteractionPotentialCollisionHandler (fixture ipm_ref_40Td.npz, 65,536
    ions x 30,000 steps at 40 Td): v_drift, K0, D_L, D_T within 4 combined
    standard errors, collision fraction within 4 sqrt(2 / collisions).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import mlp as omlp
import oracle as orc
from helpers import assert_transport_close, config0_ions, ipm_reference_case, oracle_state
from icarion_b200 import _capi as capi
from icarion_b200 import config as cfg
from icarion_b200 import ipm
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu
EV = 1.602176634e-19
AMU = 1.66053906660e-27


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def _ensemble(setup, en_td=40.0, dt=2e-10):
    domain = {"instrument": "IMS", "geometry": {"origin_m": [0.0, 0.0, -0.01], "length_m": 0.1, "radius_m": 0.05},
              "env": {"temperature_K": 300.0, "pressure_Pa": 1000.0, "gas_species": "N2"},
              "fields": {"DC": {"EN_Td": en_td}}}
    return cfg.ensemble_params(domain, 0.0, dt, detector_z_m=1e30, ipm_bmax_m=setup.b_max_m)


def test_quadrature_matches_trajectory_integrator():
    s = ipm.IpmSetup()
    c12, c6, c4 = s.coefficients()
    mu = 300 * 28.0134 / 328.0134 * AMU
    E = np.repeat(np.array([10, 26, 50, 100, 300, 1000, 3000, 10000]) * 1e-3 * EV, 13)
    b = np.tile(np.arange(13) * 1e-10, 8)
    got = ipm.deflection(s, E, b)
    want = np.array([orc.ipm_cos_chi_trajectory(c12, c6, c4, mu, e, bb) for e, bb in zip(E, b)])
    assert np.max(np.abs(got - want)) <= 1e-3, np.max(np.abs(got - want))


def test_handle_table_equals_quadrature_at_nodes():
    s = ipm.IpmSetup(n_E=64, n_b=32)
    with Simulation([_ensemble(s)], precision=capi.PREC_FP64, collision=capi.COLLISION_IPM_TABLE) as sim:
        sim.upload(config0_ions(64))
        sim.configure_ipm(s)
        tab = sim.ipm_table()
    En, bn = s.table_grid()
    E = np.repeat(En, s.n_b)
    b = np.tile(bn, s.n_E)
    want = ipm.deflection(s, E, b).reshape(s.n_E, s.n_b)
    np.testing.assert_allclose(tab, want.astype(np.float32), rtol=0, atol=2e-6)


def test_fp64_table_collisions_match_oracle():
    s = ipm.IpmSetup(n_E=128, n_b=64)
    e = _ensemble(s)
    n, steps = 512, 2000
    st0 = config0_ions(n)
    with Simulation([e], precision=capi.PREC_FP64, collision=capi.COLLISION_IPM_TABLE, rng_seed=123) as sim:
        sim.upload(st0)
        sim.configure_ipm(s)
        tab = sim.ipm_table()
        rs = sim.advance(steps)
        out = sim.download()
    orc.set_ipm_table(tab.ravel(), s.n_E, s.n_b, *s.table_scale())
    ost = oracle_state(st0)
    r = orc.run(e, ost, steps, integrator=0, collision=4, seed=123)
    pos = np.stack([out.x, out.y, out.z])
    opos = np.stack([ost["x"], ost["y"], ost["z"]])
    vel = np.stack([out.vx, out.vy, out.vz])
    ovel = np.stack([ost["vx"], ost["vy"], ost["vz"]])
    rel = np.maximum(np.linalg.norm(pos - opos, axis=0) / np.linalg.norm(opos, axis=0),
                     np.linalg.norm(vel - ovel, axis=0) / np.linalg.norm(ovel, axis=0))
    assert float(np.mean(rel < 1e-9)) >= 0.99, np.sort(rel)[-5:]
    assert abs(rs["collisions"] - r["collisions"]) <= 0.01 * r["collisions"]
    assert r["collisions"] > 0.05 * n * steps


def test_mlp_gradients_and_forward_match_numpy():
    rng = np.random.default_rng(4)
    p = ipm.init_params(11)
    p[128:192] = rng.normal(0, 0.2, 64)
    p[4288:4352] = rng.normal(0, 0.2, 64)
    x = rng.uniform(-1, 1, (4096, 2)).astype(np.float32)
    y = rng.uniform(-1, 1, 4096).astype(np.float32)
    g, loss = ipm.gradients(p, x.ravel(), y)
    l64, g64 = omlp.loss_and_grad(p.astype(np.float64), x.astype(np.float64), y.astype(np.float64))
    assert abs(loss - l64) <= 1e-5 * l64
    assert np.linalg.norm(g - g64) <= 1e-4 * np.linalg.norm(g64)
    f32 = ipm.forward(p, x.ravel(), mode=0)
    ref = omlp.forward(p.astype(np.float64), x.astype(np.float64))
    assert np.max(np.abs(f32 - ref)) <= 1e-5
    mma = ipm.forward(p, x.ravel(), mode=1)
    assert np.max(np.abs(mma - ref)) <= 2e-2 * max(1.0, np.max(np.abs(ref)))
    # partial warps: every row count 1..32 evaluates the right rows
    for n in (1, 7, 16, 17, 31, 33):
        part = ipm.forward(p, x[:n].ravel(), mode=1)
        np.testing.assert_array_equal(part, mma[:n])


def test_training_fits_the_deflection_function():
    s = ipm.IpmSetup()
    x, y, _, _ = ipm.training_set(s, n=1 << 16, seed=3)
    p, losses = ipm.train(x, y, epochs=20, batch=512, lr=3e-3, seed=5)
    assert losses[-1] < 0.1 * losses[0]
    xv, yv, _, _ = ipm.training_set(s, n=1 << 14, seed=4)
    pred = ipm.forward(p, xv, mode=1)
    assert float(np.sqrt(np.mean((pred - yv) ** 2))) < 0.15


def test_learned_deflection_drift_close_to_table():
    s = ipm.IpmSetup()
    x, y, _, _ = ipm.training_set(s, n=1 << 17, seed=3)
    p, _ = ipm.train(x, y, epochs=20, batch=1024, lr=3e-3, seed=5)
    e = _ensemble(s)
    st0 = config0_ions(20000)
    dz, finals = {}, {}
    for model in (capi.COLLISION_IPM_TABLE, capi.COLLISION_IPM_MLP):
        with Simulation([e], precision=capi.PREC_MIXED, collision=model, rng_seed=9) as sim:
            sim.upload(st0)
            sim.configure_ipm(s)
            if model == capi.COLLISION_IPM_MLP:
                sim.set_mlp(p)
            rs = sim.advance(4000)
            out = sim.download()
            assert rs["collisions"] > 0
        dz[model] = float(np.mean(out.z - st0.z))
        finals[model] = out
    assert abs(dz[capi.COLLISION_IPM_MLP] / dz[capi.COLLISION_IPM_TABLE] - 1.0) < 0.03, dz
    # the network, not the table fallback, deflected the collisions
    assert not np.array_equal(finals[capi.COLLISION_IPM_MLP].vz, finals[capi.COLLISION_IPM_TABLE].vz)


def test_mixed_precision_table_collisions_track_fp64():
    """Energies in the float path (E = mu g^2 / 2 with mu = m_i m_n / (m_i +
    m_n) formed without underflow): drift and collision count of the mixed
    form within 4 standard errors / 1 % of FP64."""
    s = ipm.IpmSetup()
    e = _ensemble(s)
    st0 = config0_ions(20000)
    res = {}
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        with Simulation([e], precision=prec, collision=capi.COLLISION_IPM_TABLE, rng_seed=9) as sim:
            sim.upload(st0)
            sim.configure_ipm(s)
            rs = sim.advance(3000)
            res[prec] = (sim.download(), rs["collisions"])
    dz64 = res[capi.PREC_FP64][0].z - st0.z
    dzm = res[capi.PREC_MIXED][0].z - st0.z
    assert abs(dzm.mean() - dz64.mean()) <= 4 * dz64.std() / np.sqrt(dz64.size)
    assert abs(res[capi.PREC_MIXED][1] / res[capi.PREC_FP64][1] - 1.0) < 0.01


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_table_collisions_match_reference_handler(golden, precision):
    """The device table path against the reference's runtime sampler (the
    same fixture pins the oracle on the CPU, tests/test_oracle_ipm_reference.py)."""
    z = golden("ipm_ref_40Td.npz")
    setup, e, st0, fit = ipm_reference_case(z)
    n, steps = int(z["n_ions"]), int(z["steps"])
    with Simulation([e], precision=precision, collision=capi.COLLISION_IPM_TABLE, rng_seed=int(z["seed"])) as sim:
        sim.upload(st0)
        sim.configure_ipm(setup)
        _, mom, tot = sim.run(steps, int(z["snap_every"]), ref_step=int(z["ref_step"]))
    assert_transport_close(fit(mom[:, 0, :]), fit(z["moments"]))
    c_ref = float(z["collisions"])
    assert abs(tot["collisions"] / c_ref - 1.0) <= 4.0 * math.sqrt(2.0 / c_ref), (tot["collisions"], c_ref)
