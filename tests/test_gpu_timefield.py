"""Time-dependent fields on the device: waveform-driven voltages
(ValueOrWaveform, all eight waveform types) and the TIMS axial field model,
through the C ABI (icb_set_waveform, icb_set_tims_field), against fixtures
made by the reference's own code and against the oracle."""
from __future__ import annotations

import json

import numpy as np
import pytest

import oracle as orc
from helpers import (apply_time_field, config0_ions, domain_json, ensemble_from_golden, golden_state,
                     oracle_state, oracle_time_field, time_field_structs)
from icarion_b200 import _capi as capi
from icarion_b200 import config as cfg
from icarion_b200._capi import IcbError
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu

TIMED_PUSHES = ["boris_tims", "rk4_tims_exp", "boris_tims_wave", "boris_lqit_wave", "rk4_ims_waveref",
                "boris_quadrf_waveref", "boris_ims_inline", "boris_lqit_ac", "rk4_lqit1_ac"]


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def vec_rel_err(out, z) -> float:
    worst = 0.0
    for grp in (("x", "y", "z"), ("vx", "vy", "vz")):
        a = np.stack([getattr(out, k) for k in grp])
        b = np.stack([z["out_" + k] for k in grp])
        scale = np.maximum(np.linalg.norm(b, axis=0), 1e-300)
        worst = max(worst, float(np.max(np.linalg.norm(a - b, axis=0) / scale)))
    return worst


def run_timed(z, precision, **kw):
    dom = json.loads(str(z["domain"]))
    integ = capi.INTEGRATOR_BORIS if str(z["integrator"]) == "boris" else capi.INTEGRATOR_RK4
    with Simulation([ensemble_from_golden(z)], precision=precision, integrator=integ,
                    collision=capi.COLLISION_NONE, **kw) as sim:
        apply_time_field(sim, dom)
        sim.upload(golden_state(z))
        sim.advance(int(z["steps"]))
        return sim.download()


@pytest.mark.parametrize("case", TIMED_PUSHES)
def test_fp64_timed_push_matches_reference(golden, case):
    """FP64 device push through waveform / TIMS fields within 1e-12 of the
    reference's own code (device sin / cos / exp against glibc's), same
    survivors."""
    z = golden(f"push_{case}.npz")
    out = run_timed(z, capi.PREC_FP64)
    assert vec_rel_err(out, z) <= 1e-12
    assert np.array_equal(out.active, z["out_active"].astype(np.uint8))


@pytest.mark.parametrize("case", TIMED_PUSHES)
def test_mixed_timed_push_close_to_reference(golden, case):
    z = golden(f"push_{case}.npz")
    assert vec_rel_err(run_timed(z, capi.PREC_MIXED), z) <= 2e-3
    if str(z["integrator"]) == "boris":
        assert vec_rel_err(run_timed(z, capi.PREC_MIXED_HILO), z) <= 2e-3


def test_fp64_tims_collisions_match_oracle():
    """TIMS profile ramp with RF confinement and HSS in N2 at 300 Pa: FP64
    device vs oracle (same skip clock, same field bound) >= 99 % of ions to
    1e-9 after 3000 steps, collision counts within 1 %; the mixed form's
    count within 1 % of FP64."""
    kw = dict(instrument="TIMS", origin_z=-0.01, length=0.02, radius=0.005, T=300, P=300.0, gas="N2",
              rf_V=180.0, rf_f=2.0e6, tims=1, tims_z="0,0.008,0.02", tims_pi="0,-800,-1500",
              tims_pf="0,-200,-300", tims_t0=5e-7, tims_t1=2.5e-6, wave_rff="4|0|0|2e6,1e5,3e5,0")
    e = cfg.ensemble_params(domain_json(kw), 150e-20, 1e-9)
    assert e["instrument"] == capi.INSTRUMENT_TIMS
    n, steps = 512, 3000
    st0 = config0_ions(n)
    st0.x *= 0.2; st0.y *= 0.2; st0.z *= 0.2
    ost = oracle_state(st0)
    r = orc.run(e, ost, steps, integrator=0, collision=2, seed=123, time_field=oracle_time_field(kw))
    outs = {}
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        with Simulation([e], precision=prec, integrator=capi.INTEGRATOR_BORIS, collision=capi.COLLISION_HSS,
                        rng_seed=123) as sim:
            apply_time_field(sim, kw)
            sim.upload(st0)
            rs = sim.advance(steps)
            outs[prec] = (sim.download(), rs)
    out, rs = outs[capi.PREC_FP64]
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
    assert abs(outs[capi.PREC_MIXED][1]["collisions"] / rs["collisions"] - 1.0) < 0.01


def test_cleared_waveform_restores_constant_field(golden):
    """Setting and clearing a waveform leaves the constant-voltage push
    (bit-identical to the fixture of the plain LQIT)."""
    z = golden("push_boris_lqit.npz")
    w, _ = time_field_structs({"wave_axial": "1|1|0|2,5,0,4e-6"})
    with Simulation([ensemble_from_golden(z)], precision=capi.PREC_FP64, integrator=capi.INTEGRATOR_BORIS,
                    collision=capi.COLLISION_NONE) as sim:
        sim.set_waveform(0, capi.CHANNEL_DC_AXIAL_V, w[capi.CHANNEL_DC_AXIAL_V])
        sim.set_waveform(0, capi.CHANNEL_DC_AXIAL_V, None)
        sim.upload(golden_state(z))
        sim.advance(int(z["steps"]))
        out = sim.download()
    assert vec_rel_err(out, z) <= 1e-12


def test_time_field_argument_checks(golden):
    """Rejected before anything runs: waveforms on the FTICR (read once at
    t = 0), the TIMS ramp channel off a TIMS domain, unbounded or malformed
    waveforms, TIMS fields on other instruments, bad profiles."""
    zf = golden("push_boris_fticr.npz")
    with Simulation([ensemble_from_golden(zf)], precision=capi.PREC_FP64, integrator=capi.INTEGRATOR_BORIS,
                    collision=capi.COLLISION_NONE) as sim:
        w = capi.Waveform()
        with pytest.raises(IcbError) as ei:
            sim.set_waveform(0, capi.CHANNEL_RF_VOLTAGE_V, w)
        assert ei.value.code == capi.ICB_ERR_UNSUPPORTED
    z = golden("push_boris_lqit.npz")
    with Simulation([ensemble_from_golden(z)], precision=capi.PREC_FP64, integrator=capi.INTEGRATOR_BORIS,
                    collision=capi.COLLISION_NONE) as sim:
        bad = []
        w = capi.Waveform(); w.type = capi.WAVE_EXPONENTIAL; w.p[:5] = [0.0, 1.0, 1e3, 0.0, 1e9]
        bad.append((capi.CHANNEL_DC_AXIAL_V, w))              # exp(1e12): unbounded
        w = capi.Waveform(); w.type = capi.WAVE_ARBITRARY; w.n_points = 3
        w.times_s[:3] = [0.0, 2.0, 1.0]; w.values[:3] = [1.0, 2.0, 3.0]
        bad.append((capi.CHANNEL_DC_QUAD_V, w))               # times not ascending
        w = capi.Waveform(); w.type = 9
        bad.append((capi.CHANNEL_RF_VOLTAGE_V, w))            # unknown type
        w = capi.Waveform(); w.type = capi.WAVE_CONSTANT; w.p[0] = float("nan")
        bad.append((capi.CHANNEL_RF_FREQUENCY_HZ, w))         # not finite
        w = capi.Waveform()
        bad.append((capi.CHANNEL_TIMS_RAMP_FRACTION, w))      # not a TIMS domain
        bad.append((capi.N_CHANNELS, w))                      # unknown channel
        for ch, w in bad:
            with pytest.raises(IcbError) as ei:
                sim.set_waveform(0, ch, w)
            assert ei.value.code == capi.ICB_ERR_INVALID_ARGUMENT, ch
        with pytest.raises(IcbError):
            sim.set_tims_field(0, capi.TimsField())
    z1 = golden("push_rk4_lqit1.npz")              # single-axis AC drive
    with Simulation([ensemble_from_golden(z1)], precision=capi.PREC_FP64, integrator=capi.INTEGRATOR_RK4,
                    collision=capi.COLLISION_NONE) as sim:
        w = capi.Waveform()
        for ch in (capi.CHANNEL_AC_X_RAMP, capi.CHANNEL_AC_Y_AMPLITUDE_V):
            with pytest.raises(IcbError) as ei:
                sim.set_waveform(0, ch, w)
            assert ei.value.code == capi.ICB_ERR_INVALID_ARGUMENT
        sim.set_waveform(0, capi.CHANNEL_AC_X_FREQUENCY_HZ, w)
    zt = golden("push_boris_tims.npz")
    with Simulation([ensemble_from_golden(zt)], precision=capi.PREC_FP64, integrator=capi.INTEGRATOR_BORIS,
                    collision=capi.COLLISION_NONE) as sim:
        with pytest.raises(IcbError):
            sim.set_waveform(0, capi.CHANNEL_AC_X_AMPLITUDE_V, capi.Waveform())
        f = capi.TimsField(); f.n_nodes = 1
        with pytest.raises(IcbError):
            sim.set_tims_field(0, f)
        f = capi.TimsField(); f.n_nodes = 2; f.z_positions_m[:2] = [0.02, 0.0]
        with pytest.raises(IcbError):
            sim.set_tims_field(0, f)
        f = capi.TimsField(); f.ramp_mode = capi.TIMS_RAMP_EXPONENTIAL; f.ramp_tau_s = 0.0
        with pytest.raises(IcbError):
            sim.set_tims_field(0, f)
        f = capi.TimsField(); f.ramp_start_s = 2.0; f.ramp_end_s = 1.0
        with pytest.raises(IcbError):
            sim.set_tims_field(0, f)
        sim.set_tims_field(0, None)


TIMS_HSS = dict(instrument="TIMS", origin_z=-0.01, length=0.02, radius=0.005, T=300, P=300.0, gas="N2",
                rf_V=180.0, rf_f=2.0e6, tims=1, tims_z="0,0.008,0.02", tims_pi="0,-800,-1500",
                tims_pf="0,-200,-300", tims_t0=5e-7, tims_t1=2.5e-6, wave_rff="4|0|0|2e6,1e5,3e5,0")


def _time_field_case(case: str, golden):
    """(ensemble, harness keys, initial state, integrator, collision model)
    of a time-dependent field case: the TIMS ramp with HSS collisions
    (Boris), or a golden LQIT push with a waveform-scanned AC drive (RK4,
    which reads the per-step field table at half steps too)."""
    if case == "tims_hss":
        e = cfg.ensemble_params(domain_json(TIMS_HSS), 150e-20, 1e-9)
        st0 = config0_ions(2000)
        st0.x *= 0.2; st0.y *= 0.2; st0.z *= 0.2
        return e, TIMS_HSS, st0, capi.INTEGRATOR_BORIS, capi.COLLISION_HSS
    z = golden(f"push_{case}.npz")
    integ = capi.INTEGRATOR_BORIS if str(z["integrator"]) == "boris" else capi.INTEGRATOR_RK4
    return ensemble_from_golden(z), json.loads(str(z["domain"])), golden_state(z), integ, capi.COLLISION_NONE


def _same_state(a, b) -> None:
    for k in ("x", "y", "z", "vx", "vy", "vz", "active"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


@pytest.mark.parametrize("case", ["tims_hss", "rk4_lqit1_ac", "boris_lqit_ac"])
def test_fp64_time_field_host_path_equals_separate_calls(golden, case):
    """icb_advance_host (4 overlapped ion chunks; the per-step field table
    built once on the copy stream for every chunk) gives the state of
    icb_update_state + icb_advance + icb_download_ions bit for bit, call
    after call."""
    e, kw, st0, integ, coll = _time_field_case(case, golden)
    args = dict(precision=capi.PREC_FP64, integrator=integ, collision=coll, rng_seed=123, steps_per_launch=128)
    with Simulation([e], **args) as sim:
        apply_time_field(sim, kw)
        sim.upload(st0)
        host = st0.copy()
        host.t_death = host.t_arrival = None
        for _ in range(3):
            sim.advance_host(host, 300, n_chunks=4)
        c_host = sim.clock()
    with Simulation([e], **args) as sim:
        apply_time_field(sim, kw)
        sim.upload(st0)
        sep = st0.copy()
        for _ in range(3):
            sim.update_state(sep)
            sim.advance(300)
            sep = sim.download(sep)
        c_sep = sim.clock()
    _same_state(host, sep)
    assert c_host[0] == c_sep[0] == 900 and np.array_equal(c_host[1], c_sep[1])


@pytest.mark.parametrize("case", ["tims_hss", "rk4_lqit1_ac"])
def test_fp64_time_field_graph_replay_equals_direct_launches(golden, case):
    """use_graphs = 1 (the field table rebuilt inside each captured launch
    sequence, replayed for repeated step counts, recaptured when the count
    changes) gives the direct-launch result bit for bit."""
    e, kw, st0, integ, coll = _time_field_case(case, golden)
    outs = []
    for graphs in (0, 1):
        with Simulation([e], precision=capi.PREC_FP64, integrator=integ, collision=coll, rng_seed=123,
                        steps_per_launch=128, use_graphs=graphs) as sim:
            apply_time_field(sim, kw)
            sim.upload(st0)
            stats = [sim.advance(k) for k in (300, 300, 125, 300)]
            outs.append((sim.download(), sim.clock(), [s["collisions"] for s in stats]))
    _same_state(outs[0][0], outs[1][0])
    assert outs[0][1][0] == outs[1][1][0] == 1025 and np.array_equal(outs[0][1][1], outs[1][1][1])
    assert outs[0][2] == outs[1][2]
