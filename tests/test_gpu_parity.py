"""Device parity through the C ABI against the reference's own outputs and
the CPU oracle.

Tolerances (stated per test):
  * FP64 collision-free push: <= 1e-12 relative; the
    uniform-field and linear-field cases are additionally bit-identical.
  * FP64 null-collision HSS vs the FP64 oracle with the same Philox streams:
    >= 99% of ions agree to 1e-9 relative after 3000 steps (transcendental
    functions differ by an ulp between CUDA and glibc, which can flip a rare
    accept/reject decision).
  * Mixed precision push: <= 1e-4 (IMS) / 2e-3 (FT-ICR, RF) relative.  The
    collision-free IMS cases accelerate v_z to ~6 km/s over 5000 steps of
    ~1 m/s, so FP32 velocity rounding accumulates to a few 1e-5.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from helpers import config0_ensemble, config0_ions, ensemble_from_golden, golden_state, oracle_state
from icarion_b200 import _capi as capi
from icarion_b200.sim import IonState, Simulation, device_count

pytestmark = pytest.mark.gpu

PUSH_CASES = ["boris_ims", "rk4_ims", "boris_fticr", "rk4_fticr", "boris_quadrf", "boris_lqit", "rk4_lqit1"]
BIT_EXACT = {"boris_ims", "rk4_ims", "boris_fticr", "rk4_fticr"}
KEYS = ("x", "y", "z", "vx", "vy", "vz")


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def vec_rel_err(out: IonState, z, prefix="out_") -> float:
    """max over ions of |a - b| / |b| per 3-vector (position and velocity)."""
    worst = 0.0
    for grp in (("x", "y", "z"), ("vx", "vy", "vz")):
        a = np.stack([getattr(out, k) for k in grp])
        b = np.stack([z[prefix + k] for k in grp])
        scale = np.maximum(np.linalg.norm(b, axis=0), 1e-300)
        worst = max(worst, float(np.max(np.linalg.norm(a - b, axis=0) / scale)))
    return worst


def run_push(z, precision, integrator) -> IonState:
    e = ensemble_from_golden(z)
    with Simulation([e], precision=precision, integrator=integrator, collision=capi.COLLISION_NONE) as sim:
        sim.upload(golden_state(z))
        sim.advance(int(z["steps"]))
        return sim.download()


@pytest.mark.parametrize("case", PUSH_CASES)
def test_fp64_push_matches_reference(golden, case):
    z = golden(f"push_{case}.npz")
    integ = capi.INTEGRATOR_BORIS if case.startswith("boris") else capi.INTEGRATOR_RK4
    out = run_push(z, capi.PREC_FP64, integ)
    err = vec_rel_err(out, z)
    assert err <= 1e-12, err
    if case in BIT_EXACT:
        for k in KEYS:
            assert np.array_equal(getattr(out, k), z[f"out_{k}"]), k
    assert np.array_equal(out.active, z["out_active"].astype(np.uint8))


@pytest.mark.parametrize("case", PUSH_CASES)
def test_mixed_push_close_to_reference(golden, case):
    z = golden(f"push_{case}.npz")
    integ = capi.INTEGRATOR_BORIS if case.startswith("boris") else capi.INTEGRATOR_RK4
    tol = 1e-4 if case.endswith("ims") else 2e-3
    err = vec_rel_err(run_push(z, capi.PREC_MIXED, integ), z)
    assert err <= tol, err
    if case.startswith("boris"):
        err_hl = vec_rel_err(run_push(z, capi.PREC_MIXED_HILO, integ), z)
        assert err_hl <= tol, err_hl


def test_philox_device_matches_oracle_and_curand():
    rng = np.random.default_rng(11)
    n = 4096
    ctr = rng.integers(0, 2**32, size=(n, 4), dtype=np.uint64).astype(np.uint32)
    seed = 0x0123456789ABCDEF
    ref = orc.philox(ctr, seed)
    for use_curand in (0, 1):
        out = np.zeros_like(ctr)
        capi.check(capi.lib().icb_philox_eval(0, n, capi.u32ptr(np.ascontiguousarray(ctr)), seed, use_curand,
                                              capi.u32ptr(out)))
        assert np.array_equal(out, ref), f"use_curand={use_curand}"


def _hss_gpu(st0: IonState, e: dict, steps: int, **kw) -> tuple[IonState, dict]:
    with Simulation([e], precision=kw.pop("precision", capi.PREC_FP64), integrator=capi.INTEGRATOR_BORIS,
                    collision=kw.pop("collision", capi.COLLISION_HSS), rng_seed=123, **kw) as sim:
        sim.upload(st0)
        rs = sim.advance(steps)
        return sim.download(), rs


def _clock_math(x, which):
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    capi.check(capi.lib().icb_clock_math_eval(0, x.size, capi.fptr(x), which, capi.fptr(out)))
    return out.astype(np.float64)


def test_float_clock_functions_match_cuda():
    """The float kernels' -ln(1 - q) and 1 - e^-x (Taylor series below 1/4,
    hardware log/exp above) against CUDA's log1pf / expm1f on the device and
    against FP64: relative error <= 3e-7 on the series range, <= 2e-6 on
    the rest (q up to the kernel's cap 1 - 2^-20, x up to 30)."""
    q = np.concatenate([np.logspace(-12, np.log10(0.2499), 4000), np.linspace(0.25, 0.99999904632568359375, 4000)])
    q = q.astype(np.float32).astype(np.float64)
    exact = -np.log1p(-q)
    ours, cuda = _clock_math(q, capi.MATH_NEG_LOG1M), _clock_math(q, capi.MATH_NEG_LOG1M_CUDA)
    lo = q < 0.25
    for got in (ours, cuda):
        rel = np.abs(got - exact) / exact
        assert rel[lo].max() <= 3e-7 and rel[~lo].max() <= 2e-6, (rel[lo].max(), rel[~lo].max())
    assert np.max(np.abs(ours - cuda) / exact) <= 2e-6
    x = np.concatenate([np.logspace(-12, np.log10(0.2499), 4000), np.linspace(0.25, 30.0, 4000)])
    x = x.astype(np.float32).astype(np.float64)
    exact = -np.expm1(-x)
    ours, cuda = _clock_math(x, capi.MATH_ONE_MINUS_EXP), _clock_math(x, capi.MATH_ONE_MINUS_EXP_CUDA)
    lo = x < 0.25
    for got in (ours, cuda):
        rel = np.abs(got - exact) / exact
        assert rel[lo].max() <= 3e-7 and rel[~lo].max() <= 2e-6, (rel[lo].max(), rel[~lo].max())
    with pytest.raises(capi.IcbError):
        _clock_math(x[:4], 9)


def test_fp64_hss_trajectories_match_oracle():
    n, steps = 512, 3000
    e = config0_ensemble()
    st0 = config0_ions(n)
    ost = oracle_state(st0)
    r = orc.run(e, ost, steps, integrator=0, collision=2, seed=123)
    out, rs = _hss_gpu(st0, e, steps)
    pos = np.stack([out.x, out.y, out.z])
    opos = np.stack([ost["x"], ost["y"], ost["z"]])
    vel = np.stack([out.vx, out.vy, out.vz])
    ovel = np.stack([ost["vx"], ost["vy"], ost["vz"]])
    rel = np.maximum(np.linalg.norm(pos - opos, axis=0) / np.linalg.norm(opos, axis=0),
                     np.linalg.norm(vel - ovel, axis=0) / np.linalg.norm(ovel, axis=0))
    frac = float(np.mean(rel < 1e-9))
    assert frac >= 0.99, (frac, np.sort(rel)[-5:])
    assert abs(rs["collisions"] - r["collisions"]) <= 0.01 * r["collisions"]
    assert r["collisions"] > 0.05 * n * steps      # ~9% of ion-steps collide at config 0


def test_fp64_langevin_trajectories_match_oracle():
    """Langevin capture collisions (constant rate per ion, Maxwellian
    neutral, isotropic COM scatter) against the oracle with the same Philox
    streams: >= 99 % of ions to 1e-9 after 3000 steps; same collision count
    within 1 %."""
    n, steps = 512, 3000
    e = config0_ensemble()
    st0 = config0_ions(n)
    ost = oracle_state(st0)
    r = orc.run(e, ost, steps, integrator=0, collision=3, seed=123)
    out, rs = _hss_gpu(st0, e, steps, collision=capi.COLLISION_LANGEVIN)
    pos = np.stack([out.x, out.y, out.z])
    opos = np.stack([ost["x"], ost["y"], ost["z"]])
    vel = np.stack([out.vx, out.vy, out.vz])
    ovel = np.stack([ost["vx"], ost["vy"], ost["vz"]])
    rel = np.maximum(np.linalg.norm(pos - opos, axis=0) / np.linalg.norm(opos, axis=0),
                     np.linalg.norm(vel - ovel, axis=0) / np.linalg.norm(ovel, axis=0))
    assert float(np.mean(rel < 1e-9)) >= 0.99, np.sort(rel)[-5:]
    assert abs(rs["collisions"] - r["collisions"]) <= 0.01 * r["collisions"]
    assert r["collisions"] == r["candidates"] > 0.02 * n * steps


MIX2 = [("N2", 0.79, 150e-20), ("He", 0.21, 60e-20)]
MIX7 = [("N2", 0.50, 150e-20), ("He", 0.14, 60e-20), ("Ar", 0.10, 130e-20), ("O2", 0.09, 140e-20),
        ("CO2", 0.07, 190e-20), ("Ne", 0.06, 80e-20), ("H2O", 0.04, 120e-20)]


@pytest.mark.parametrize("mix_def", [MIX2, MIX7], ids=["2 gases", "7 gases"])
def test_fp64_gas_mixture_trajectories_match_oracle(mix_def):
    """HSS in a gas mixture (HSSCollisionHandler.cpp:105-249) against the
    oracle's restatement with the same Philox streams (the oracle itself is
    checked against the reference handler on CPU): >= 99 % of ions to 1e-9
    after 3000 steps, collision counts within 1 %; mixed precision keeps the
    collision fraction within 1 % and the drift within 4 standard errors."""
    from icarion_b200 import config as cfg
    from helpers import CONFIG0_DOMAIN, domain_json
    dom = domain_json(CONFIG0_DOMAIN)
    dom["env"]["gas_mixture"] = [{"species": g, "mole_fraction": f, "cross_section_m2": c} for g, f, c in mix_def]
    e = cfg.ensemble_params(dom, 150e-20, 5e-10)
    n, steps = 512, 3000
    st0 = config0_ions(n)
    ost = oracle_state(st0)
    r = orc.run(e, ost, steps, integrator=0, collision=5, seed=123)
    out, rs = _hss_gpu(st0, e, steps)
    pos = np.stack([out.x, out.y, out.z])
    opos = np.stack([ost["x"], ost["y"], ost["z"]])
    vel = np.stack([out.vx, out.vy, out.vz])
    ovel = np.stack([ost["vx"], ost["vy"], ost["vz"]])
    rel = np.maximum(np.linalg.norm(pos - opos, axis=0) / np.linalg.norm(opos, axis=0),
                     np.linalg.norm(vel - ovel, axis=0) / np.linalg.norm(ovel, axis=0))
    assert float(np.mean(rel < 1e-9)) >= 0.99, np.sort(rel)[-5:]
    assert abs(rs["collisions"] - r["collisions"]) <= 0.01 * r["collisions"]
    st1 = config0_ions(8192)
    f64, r64 = _hss_gpu(st1, e, steps)
    mix, rmx = _hss_gpu(st1, e, steps, precision=capi.PREC_MIXED)
    assert abs(rmx["collisions"] / r64["collisions"] - 1.0) < 0.01
    dz64, dzm = f64.z - st1.z, mix.z - st1.z
    assert abs(dzm.mean() - dz64.mean()) <= 4 * dz64.std() / np.sqrt(8192)


@pytest.mark.parametrize("model", ["axial_parabolic", "axial_uniform"])
def test_fp64_gas_flow_trajectories_match_oracle(model):
    """Gas flow evaluated at the colliding ion (EnvironmentConfig.h:96-128;
    the oracle itself is checked against the reference's flow and handler on
    CPU): FP64 device vs oracle >= 99 % of ions to 1e-9 after 3000 steps,
    collision counts within 1 %; the float forms keep the collision
    fraction within 1 % and the mean drift within 4 standard errors."""
    from test_oracle_flow import CASES, flow_ensemble
    e = flow_ensemble(model, CASES[model][0])
    n, steps = 512, 3000
    st0 = config0_ions(n)
    ost = oracle_state(st0)
    r = orc.run(e, ost, steps, integrator=0, collision=2, seed=123)
    out, rs = _hss_gpu(st0, e, steps)
    live = (ost["active"] != 0) & (out.active != 0)
    assert live.sum() > 0.8 * n and np.array_equal(ost["active"] != 0, out.active != 0)
    pos = np.stack([out.x, out.y, out.z])[:, live]
    opos = np.stack([ost["x"], ost["y"], ost["z"]])[:, live]
    vel = np.stack([out.vx, out.vy, out.vz])[:, live]
    ovel = np.stack([ost["vx"], ost["vy"], ost["vz"]])[:, live]
    rel = np.maximum(np.linalg.norm(pos - opos, axis=0) / np.linalg.norm(opos, axis=0),
                     np.linalg.norm(vel - ovel, axis=0) / np.linalg.norm(ovel, axis=0))
    assert float(np.mean(rel < 1e-9)) >= 0.99, np.sort(rel)[-5:]
    assert abs(rs["collisions"] - r["collisions"]) <= 0.01 * r["collisions"]
    st1 = config0_ions(8192)
    f64, r64 = _hss_gpu(st1, e, steps)
    for prec in (capi.PREC_MIXED, capi.PREC_MIXED_HILO):
        mix, rmx = _hss_gpu(st1, e, steps, precision=prec)
        assert abs(rmx["collisions"] / r64["collisions"] - 1.0) < 0.01
        a64, am = f64.active != 0, mix.active != 0
        dz64, dzm = (f64.z - st1.z)[a64], (mix.z - st1.z)[am]
        assert abs(dzm.mean() - dz64.mean()) <= 4 * dz64.std() / np.sqrt(dz64.size)


def test_fp64_lqit_collisions_match_oracle():
    """Linear ion trap (RF quadrupole about the axis, axial DC well, two-axis
    dipolar drive; AnalyticalFieldModel.cpp:81-134) with HSS in He at 50 Pa:
    FP64 device vs oracle >= 99 % of ions to 1e-9 after 3000 steps, collision
    counts within 1 %; the mixed form's collision count within 1 % of FP64."""
    from helpers import domain_json
    from icarion_b200 import config as cfg
    kw = dict(instrument="LQIT", origin_z=-0.025, length=0.05, radius=0.004, T=300, P=50.0, gas="He",
              rf_V=200.0, rf_f=1.0e6, dc_quad_V=1.0, axial_V=2.0,
              dip_x_A=0.5, dip_x_f=1.0e5, dip_x_phase=0.3, dip_x_ramp=0.8, dip_y_A=0.2, dip_y_f=1.2e5)
    e = cfg.ensemble_params(domain_json(kw), 150e-20, 1e-9)
    assert e["instrument"] == capi.INSTRUMENT_LQIT and e["ac_dipolar"] == 1
    n, steps = 512, 3000
    st0 = config0_ions(n)
    st0.x *= 0.2; st0.y *= 0.2; st0.z *= 0.2
    ost = oracle_state(st0)
    r = orc.run(e, ost, steps, integrator=0, collision=2, seed=123)
    out, rs = _hss_gpu(st0, e, steps)
    assert r["collisions"] > 50 * n
    live = (ost["active"] != 0) & (out.active != 0)
    assert live.sum() > 0.9 * n
    pos = np.stack([out.x, out.y, out.z])[:, live]
    opos = np.stack([ost["x"], ost["y"], ost["z"]])[:, live]
    vel = np.stack([out.vx, out.vy, out.vz])[:, live]
    ovel = np.stack([ost["vx"], ost["vy"], ost["vz"]])[:, live]
    rel = np.maximum(np.linalg.norm(pos - opos, axis=0) / np.linalg.norm(opos, axis=0),
                     np.linalg.norm(vel - ovel, axis=0) / np.linalg.norm(ovel, axis=0))
    assert float(np.mean(rel < 1e-9)) >= 0.99, np.sort(rel)[-5:]
    assert abs(rs["collisions"] - r["collisions"]) <= 0.01 * r["collisions"]
    _, rmx = _hss_gpu(st0, e, steps, precision=capi.PREC_MIXED)
    assert abs(rmx["collisions"] / rs["collisions"] - 1.0) < 0.01


@pytest.mark.parametrize("subcycles", [1, 4])
def test_fp64_plain_form_matches_oracle(subcycles):
    """The plain per-step HSS form (the bench's plain FP64 baseline; with 4
    collision sub-steps per step) against the oracle with the same Philox
    words: >= 99 % of ions to 1e-9 after 3000 steps, collision counts within
    1 %."""
    n, steps = 512, 3000
    e = config0_ensemble()
    st0 = config0_ions(n)
    ost = oracle_state(st0)
    r = orc.run(e, ost, steps, integrator=0, collision=6, seed=123, subcycles=subcycles)
    out, rs = _hss_gpu(st0, e, steps, collision=capi.COLLISION_HSS_PLAIN, collision_subcycles=subcycles)
    pos = np.stack([out.x, out.y, out.z])
    opos = np.stack([ost["x"], ost["y"], ost["z"]])
    vel = np.stack([out.vx, out.vy, out.vz])
    ovel = np.stack([ost["vx"], ost["vy"], ost["vz"]])
    rel = np.maximum(np.linalg.norm(pos - opos, axis=0) / np.linalg.norm(opos, axis=0),
                     np.linalg.norm(vel - ovel, axis=0) / np.linalg.norm(ovel, axis=0))
    assert float(np.mean(rel < 1e-9)) >= 0.99, np.sort(rel)[-5:]
    assert abs(rs["collisions"] - r["collisions"]) <= 0.01 * r["collisions"]
    assert rs["candidates"] == n * steps * subcycles


def test_fp64_ehss_trajectories_match_oracle():
    """EHSS collisions on a 7-atom molecule against the oracle's
    restatement (itself checked against the reference kernel on CPU): >= 99 %
    of FP64 ions to 1e-9 after 2000 steps, collision counts within 1 %; the
    mixed form's collision count within 1 % of FP64."""
    from test_oracle_ehss import molecule
    at = molecule()
    e = config0_ensemble()
    n, steps = 512, 2000
    st0 = config0_ions(n)
    ost = oracle_state(st0)
    orc.set_ehss(at, 1.8e-10)
    r = orc.run(e, ost, steps, integrator=0, collision=7, seed=123)

    def run(prec, st):
        with Simulation([e], precision=prec, collision=capi.COLLISION_EHSS, rng_seed=123) as sim:
            sim.upload(st)
            sim.set_ehss_geometry(0, at[:, :3], at[:, 3], 1.8e-10)
            rs = sim.advance(steps)
            return sim.download(), rs
    out, rs = run(capi.PREC_FP64, st0)
    pos = np.stack([out.x, out.y, out.z])
    opos = np.stack([ost["x"], ost["y"], ost["z"]])
    vel = np.stack([out.vx, out.vy, out.vz])
    ovel = np.stack([ost["vx"], ost["vy"], ost["vz"]])
    rel = np.maximum(np.linalg.norm(pos - opos, axis=0) / np.linalg.norm(opos, axis=0),
                     np.linalg.norm(vel - ovel, axis=0) / np.linalg.norm(ovel, axis=0))
    assert float(np.mean(rel < 1e-9)) >= 0.99, np.sort(rel)[-5:]
    assert abs(rs["collisions"] - r["collisions"]) <= 0.01 * r["collisions"]
    st1 = config0_ions(8192)
    _, r64 = run(capi.PREC_FP64, st1)
    _, rmx = run(capi.PREC_MIXED, st1)
    assert abs(rmx["collisions"] / r64["collisions"] - 1.0) < 0.01


def test_results_independent_of_launch_shape():
    """Same Philox counters and per-lane step order: block size, steps per
    launch and the deferred-collision threshold do not change results."""
    n, steps = 3000, 1500
    e = config0_ensemble()
    st0 = config0_ions(n)
    outs = []
    for bs, K, pend in ((128, 1000, 16), (64, 7, 1), (96, 333, 32)):
        out, _ = _hss_gpu(st0, e, steps, block_size=bs, steps_per_launch=K, pending_threshold=pend)
        outs.append(out)
    for o in outs[1:]:
        for k in KEYS:
            assert np.array_equal(getattr(o, k), getattr(outs[0], k)), k


def _chunks(st0, e, chunks, precision, **kw):
    with Simulation([e], precision=precision, integrator=capi.INTEGRATOR_BORIS, collision=capi.COLLISION_HSS,
                    rng_seed=123, **kw) as sim:
        sim.upload(st0)
        stats = [sim.advance(k) for k in chunks]
        return sim.download(), sim.clock(), stats


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_graph_replay_equals_direct_launches(precision):
    """icb_advance through a captured CUDA graph (replayed for repeated
    n_steps, recaptured when n_steps changes) gives the direct-launch result
    bit for bit, with the same counters and device clock."""
    e = config0_ensemble()
    st0 = config0_ions(3000)
    chunks = (300, 300, 300, 125, 300)
    direct, c0, s0 = _chunks(st0, e, chunks, precision, steps_per_launch=128)
    graph, c1, s1 = _chunks(st0, e, chunks, precision, steps_per_launch=128, use_graphs=1)
    for k in KEYS:
        assert np.array_equal(getattr(graph, k), getattr(direct, k)), k
    assert c0[0] == c1[0] == sum(chunks) and np.array_equal(c0[1], c1[1])
    for a, b in zip(s0, s1):
        assert (a["collisions"], a["candidates"], a["kernel_launches"]) == \
               (b["collisions"], b["candidates"], b["kernel_launches"])


def test_autotune_restores_state_and_keeps_fp64_results():
    """icb_autotune times launch shapes from a saved copy of the state and
    puts it back: an FP64 run tuned half way equals an untuned run bit for bit."""
    e = config0_ensemble()
    st0 = config0_ions(4000)
    plain, c0, _ = _chunks(st0, e, (400, 600), capi.PREC_FP64)
    with Simulation([e], precision=capi.PREC_FP64, integrator=capi.INTEGRATOR_BORIS, collision=capi.COLLISION_HSS,
                    rng_seed=123) as sim:
        sim.upload(st0)
        sim.advance(400)
        t = sim.autotune(trial_steps=200)
        assert sim.clock()[0] == 400
        sim.advance(600)
        tuned = sim.download()
        c1 = sim.clock()
    assert t["trials"] == 18 and t["block_size"] in (64, 128) and t["ion_steps_per_s"] > 0
    assert t["steps_per_vote"] in (4, 8, 16) and t["pending_threshold"] in (6, 10, 14)
    for k in KEYS:
        assert np.array_equal(getattr(tuned, k), getattr(plain, k)), k
    assert c0[0] == c1[0] and np.array_equal(c0[1], c1[1])


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_advance_host_equals_separate_calls(precision):
    """icb_advance_host with 4 overlapped ion chunks gives the state of
    icb_update_state + icb_advance + icb_download_ions bit for bit."""
    e = config0_ensemble()
    st0 = config0_ions(5000)
    outs = []
    for chunks in (1, 4):
        with Simulation([e], precision=precision, collision=capi.COLLISION_HSS, rng_seed=3,
                        steps_per_launch=400) as sim:
            sim.upload(st0)
            host = st0.copy()
            host.t_death = host.t_arrival = None
            for _ in range(3):
                rs = sim.advance_host(host, 400, n_chunks=chunks)
            outs.append((host, sim.clock(), rs["collisions"]))
    for k in KEYS + ("active",):
        assert np.array_equal(getattr(outs[0][0], k), getattr(outs[1][0], k)), k
    assert outs[0][1][0] == outs[1][1][0] == 1200 and outs[0][2] == outs[1][2]


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_advance_host_with_graphs_equals_separate_calls(precision):
    """A handle that replays icb_advance through CUDA graphs runs
    icb_advance_host as overlapped ion chunks too (plain launches), on two
    ensembles whose boundary falls inside a chunk; mixed with graph-replayed
    icb_advance calls it gives the state of the same calls without graphs
    and of icb_update_state + icb_advance + icb_download_ions, bit for bit."""
    e = config0_ensemble()
    st0 = config0_ions(5000)
    offsets = [0, 2900, 5000]
    outs = []
    for graphs, chunks in ((0, 1), (1, 4), (0, 4)):
        with Simulation([e, e], precision=precision, collision=capi.COLLISION_HSS, rng_seed=3,
                        steps_per_launch=400, use_graphs=graphs) as sim:
            sim.upload(st0, ens_offsets=offsets)
            host = st0.copy()
            host.t_death = host.t_arrival = None
            colls = 0
            for _ in range(2):
                colls += sim.advance_host(host, 400, n_chunks=chunks)["collisions"]
            sim.update_state(host)
            colls += sim.advance(400)["collisions"]
            host = sim.download(host)
            outs.append((host, sim.clock(), colls))
    for o in outs[1:]:
        for k in KEYS + ("active",):
            assert np.array_equal(getattr(outs[0][0], k), getattr(o[0], k)), k
        assert o[1][0] == outs[0][1][0] == 1200 and o[2] == outs[0][2]


def test_unfused_plug_points_equal_fused_step():
    """push (step_batch) -> collide (handle_batch) -> finalize, one call each
    per step, gives the fused icb_advance result bit for bit (FP64)."""
    n, steps = 1024, 200
    e = config0_ensemble()
    st0 = config0_ions(n)
    fused, _ = _hss_gpu(st0, e, steps)
    with Simulation([e], precision=capi.PREC_FP64, collision=capi.COLLISION_HSS, rng_seed=123) as sim:
        sim.upload(st0)
        for _ in range(steps):
            sim.step_batch()
            sim.handle_batch()
            sim.finalize()
        parts = sim.download()
        step, t = sim.clock()
    assert step == steps
    for k in KEYS:
        assert np.array_equal(getattr(parts, k), getattr(fused, k)), k


def test_domain_exit_death_times_match_oracle():
    """Ions leaving a small cylinder are deactivated with death time = start
    of the step (SimulationEngineLifecycle.cpp:139-147); FP64 vs oracle."""
    n, steps = 256, 4000
    e = config0_ensemble()
    e.update(radius_m=6e-4, length_m=2.6e-3, origin_m=[0.0, 0.0, -1.3e-3])
    st0 = config0_ions(n)
    ost = oracle_state(st0)
    orc.run(e, ost, steps, integrator=0, collision=2, seed=123)
    out, rs = _hss_gpu(st0, e, steps)
    dead = ost["active"] == 0
    assert dead.sum() > n // 4
    agree = np.mean((out.active == ost["active"]) & (out.t_death == ost["t_death"]))
    assert agree >= 0.98, agree
    assert rs["deaths"] == int(np.sum(out.active == 0))


def test_outside_and_nonfinite_ions_are_deactivated():
    e = config0_ensemble()
    st = config0_ions(64)
    st.z[3] = 0.5                 # outside the cylinder before the first step
    st.vx[5] = np.nan             # non-finite velocity
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        out, rs = _hss_gpu(st, e, 10, precision=prec)
        assert out.active[3] == 0 and out.t_death[3] == 0.0
        assert out.active[5] == 0 and out.t_death[5] == 0.0
        assert int(out.active.sum()) == 62


def test_births_wait_until_birth_time():
    e = config0_ensemble()
    st = config0_ions(32)
    st.birth = np.zeros(32)
    st.birth[:8] = 1.0            # never born within the run
    st.birth[8:16] = 50 * 5e-10   # born at step 50
    with Simulation([e], precision=capi.PREC_FP64, collision=capi.COLLISION_HSS) as sim:
        sim.upload(st)
        sim.advance(49)
        mid = sim.download()
        sim.advance(51)
        end = sim.download()
    assert np.array_equal(mid.z[:16], st.z[:16]) and not mid.active[:16].any()
    assert not end.active[:8].any() and np.array_equal(end.z[:8], st.z[:8])
    assert end.active[8:].all() and not np.array_equal(end.z[8:16], st.z[8:16])


def test_invalid_inputs_raise():
    e = config0_ensemble()
    with Simulation([e], precision=capi.PREC_MIXED) as sim:
        st = config0_ions(16)
        st.mass[2] = 0.0
        with pytest.raises(capi.IcbError):
            sim.upload(st)
        with pytest.raises(capi.IcbError):
            sim.advance(10)       # nothing uploaded
    with pytest.raises(capi.IcbError):
        Simulation([dict(e, dt_s=0.0)])
