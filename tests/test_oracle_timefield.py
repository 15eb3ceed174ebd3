"""Time-dependent fields on the CPU: the oracle's restatement of the
reference's waveforms (WaveformConfig.h / .cpp), TIMS axial field model
(TIMSAxialFieldModel.h) and the waveform-driven IMS / QuadrupoleRF / LQIT
fields against fixtures made by the reference's own code, and the JSON
adapter (config.time_fields) against the loader's rules."""
from __future__ import annotations

import json
import math

import numpy as np
import pytest

import oracle as orc
from helpers import (domain_json, ensemble_from_golden, golden_state, oracle_state, oracle_time_field,
                     time_field_structs, wave_json)
from icarion_b200 import _capi as capi
from icarion_b200 import config as cfg

TIMED_PUSHES = ["boris_tims", "rk4_tims_exp", "boris_tims_wave", "boris_lqit_wave", "rk4_ims_waveref",
                "boris_quadrf_waveref", "boris_ims_inline", "boris_lqit_ac", "rk4_lqit1_ac"]
KEYS = ("x", "y", "z", "vx", "vy", "vz")


def _field_cases(golden):
    z = golden("field_timed.npz")
    return z, json.loads(str(z["names"]))


def test_field_models_bit_exact(golden):
    """E of the restated field models equals the reference's field model
    (the one PhysicsSetup builds) at 52 (x, y, z, t) points per case: TIMS
    linear / exponential / waveform ramps and profiles, LQIT and waveform_ref
    IMS / QuadrupoleRF channels, every waveform type, and inline IMS
    waveforms read as 0 V."""
    z, names = _field_cases(golden)
    assert len(names) >= 20
    for name in names:
        kw = json.loads(str(z[f"{name}_domain"]))
        e = cfg.ensemble_params(domain_json(kw), 150e-20, 1e-9)
        E = orc.field(e, z[f"{name}_pts"], time_field=oracle_time_field(kw))
        assert np.array_equal(E, z[f"{name}_E"]), name
    # the inline-waveform IMS case really is field-free
    assert not np.any(z["ims_inline_E"])


@pytest.mark.parametrize("case", TIMED_PUSHES)
def test_timed_push_restatement_bit_exact(golden, case):
    g = golden(f"push_{case}.npz")
    kw = json.loads(str(g["domain"]))
    st = oracle_state(golden_state(g))
    orc.run(ensemble_from_golden(g), st, int(g["steps"]), integrator=0 if case.startswith("boris") else 1,
            time_field=oracle_time_field(kw))
    for k in KEYS:
        assert np.array_equal(st[k], g[f"out_{k}"]), k
    assert np.array_equal(st["active"], g["out_active"].astype(np.uint8))


def _wave_specs(golden) -> dict:
    z, names = _field_cases(golden)
    return {n: json.loads(str(z[f"{n}_domain"]))["wave_rfv"] for n in names if n.startswith("wave_")}


def test_waveform_json_adapter_matches_specs(golden):
    """config.waveform on the loader's JSON objects builds the same
    icb_waveform as the harness spec, for every type."""
    specs = _wave_specs(golden)
    assert len(specs) == 13
    for name, spec in specs.items():
        a = cfg.waveform(wave_json(spec))
        b = orc.wave_struct(spec, cls=capi.Waveform)
        assert bytes(a) == bytes(b), name


def test_host_wave_value_matches_oracle(golden):
    """The host evaluator (the FTICR radial voltage at t = 0) agrees with
    the restatement at every time of the grid, cubic tables excepted."""
    ts = np.concatenate([np.linspace(-1e-6, 8e-6, 91), [0.0, 5e-7, 1e-6, 2.5e-6, 3e-6, 4e-6, 4.1e-6]])
    for name, spec in _wave_specs(golden).items():
        if name == "wave_arbitrary_cubic":
            continue
        w = cfg.waveform(wave_json(spec))
        for t in ts:
            assert cfg.wave_value(w, float(t)) == orc.wave_value(spec, float(t)), (name, t)


def test_loader_rules():
    """WaveformLoader checks and the ValueOrWaveform forms."""
    with pytest.raises(ValueError):
        cfg.waveform({"type": "linear", "start": 0, "end": 1, "start_time_s": 1.0, "end_time_s": 1.0})
    with pytest.raises(ValueError):
        cfg.waveform({"type": "arbitrary", "times": [0, 0], "values": [1, 2]})
    with pytest.raises(ValueError):
        cfg.waveform({"type": "pwm", "low": 0, "high": 1, "frequency_Hz": 1e3, "duty_cycle": 1.5})
    with pytest.raises(ValueError):
        cfg.waveform({"type": "triangle"})
    lib = {"ramp": {"type": "linear", "start": 0, "end": 5, "end_time_s": 1e-3}}
    assert cfg.value_or_waveform(3.5, lib) == 3.5
    w = cfg.value_or_waveform("@ramp", lib)
    assert w.type == capi.WAVE_LINEAR and list(w.p[:4]) == [0.0, 5.0, 0.0, 1e-3] and w.clamp == 1
    with pytest.raises(ValueError):
        cfg.value_or_waveform("ramp", lib)
    with pytest.raises(ValueError):
        cfg.value_or_waveform("@missing", lib)


def test_time_fields_follow_the_field_models():
    """IMS / QuadrupoleRF read inline waveforms as 0 V (constant 0 in the
    ensemble, no channel); the LQIT and TIMS models evaluate them; an
    enabled TIMS block turns any instrument into the TIMS model; "@id"
    resolves through the domain's waveform library."""
    sweep = {"type": "linear", "start": 100.0, "end": 300.0, "end_time_s": 1e-3}
    for inst, expect in (("IMS", False), ("QuadrupoleRF", False), ("LQIT", True), ("TIMS", True)):
        dom = {"instrument": inst, "geometry": {"length_m": 0.05, "radius_m": 0.004},
               "env": {"temperature_K": 300.0, "pressure_Pa": 1.0, "gas_species": "He"},
               "fields": {"waveforms": {"sweep": sweep}, "RF": {"voltage_V": "@sweep", "frequency_Hz": 1e6},
                          "DC": {"axial_V": sweep}}}
        e = cfg.ensemble_params(dom, 1e-18, 1e-9)
        assert e["rf_voltage_V"] == 0.0 and e["axial_V"] == 0.0 and e["rf_frequency_Hz"] == 1e6
        waves, tims = cfg.time_fields(dom)
        assert (capi.CHANNEL_RF_VOLTAGE_V in waves) == expect, inst
        assert (capi.CHANNEL_DC_AXIAL_V in waves) == expect, inst
        assert e["instrument"] == cfg.INSTRUMENTS[inst]
        assert tims is None      # no TIMS block: a TIMS domain has a zero axial field
    # an enabled TIMS block on an IMS domain selects the TIMS model
    dom = {"instrument": "IMS", "geometry": {"length_m": 0.02, "radius_m": 0.005},
           "env": {"temperature_K": 300.0, "pressure_Pa": 300.0, "gas_species": "N2"},
           "fields": {"TIMS": {"z_positions_m": [0.0, 0.02], "axial_field_initial_profile_V_m": [0.0, -4000.0],
                               "ramp_start_s": 1e-3, "ramp_end_s": 2e-3, "ramp_fraction": 0.25}}}
    e = cfg.ensemble_params(dom, 1e-18, 1e-9)
    assert e["instrument"] == capi.INSTRUMENT_TIMS
    waves, tims = cfg.time_fields(dom)
    assert tims.n_nodes == 2 and tims.has_final_profile == 0 and tims.ramp_mode == capi.TIMS_RAMP_LINEAR
    assert list(tims.initial_profile_V_m[:2]) == [0.0, -4000.0]
    assert waves[capi.CHANNEL_TIMS_RAMP_FRACTION].type == capi.WAVE_CONSTANT
    assert waves[capi.CHANNEL_TIMS_RAMP_FRACTION].p[0] == 0.25
    # a disabled block on an IMS domain leaves the IMS model
    dom["fields"]["TIMS"]["enabled"] = False
    assert cfg.ensemble_params(dom, 1e-18, 1e-9)["instrument"] == capi.INSTRUMENT_IMS
    # FTICR reads its radial voltage once, at t = 0
    fticr = {"instrument": "FTICR", "geometry": {"length_m": 0.05, "radius_m": 0.025},
             "env": {"temperature_K": 300.0, "pressure_Pa": 1e-7, "gas_species": "He"},
             "fields": {"DC": {"radial_V": {"type": "sinusoidal", "offset": 1.0, "amplitude": 0.5,
                                            "frequency_Hz": 1e3, "phase_rad": 0.5}}}}
    assert cfg.ensemble_params(fticr, 1e-18, 1e-9)["radial_V"] == 1.0 + 0.5 * math.sin(0.5)


def test_ac_drive_channels_from_json():
    """LQIT AC drives as waveforms: dipolar axes carry amplitude, frequency
    and ramp channels, a disabled axis none; the single-axis drive carries
    amplitude and frequency (AnalyticalFieldModel.cpp:47-61, 104-121)."""
    chirp = {"type": "linear", "start": 1e5, "end": 2e5, "end_time_s": 1e-3}
    fade = {"type": "linear", "start": 0.0, "end": 1.0, "end_time_s": 1e-4}
    base = {"instrument": "LQIT", "geometry": {"length_m": 0.05, "radius_m": 0.004},
            "env": {"temperature_K": 300.0, "pressure_Pa": 0.1, "gas_species": "He"}}
    dom = dict(base, fields={"AC": {"dipolar_excitation": {
        "x": {"amplitude_V": 0.5, "frequency_Hz": chirp, "ramp": fade},
        "y": {"enabled": False, "amplitude_V": chirp}}}})
    e = cfg.ensemble_params(dom, 1e-18, 1e-9)
    assert e["ac_dipolar"] == 1 and e["ac_amplitude_V"] == [0.5, 0.0] and e["ac_frequency_Hz"][0] == 0.0
    waves, _ = cfg.time_fields(dom)
    assert set(waves) == {capi.CHANNEL_AC_X_FREQUENCY_HZ, capi.CHANNEL_AC_X_RAMP}
    dom = dict(base, fields={"AC": {"voltage_V": chirp, "frequency_Hz": 9e4}})
    waves, _ = cfg.time_fields(dom)
    assert set(waves) == {capi.CHANNEL_AC_X_AMPLITUDE_V}
    assert cfg.ensemble_params(dom, 1e-18, 1e-9)["ac_dipolar"] == 0


def test_time_field_structs_layout():
    """The ABI structs and the oracle's copies have the same size."""
    import ctypes as C
    assert C.sizeof(capi.Waveform) == C.sizeof(orc.OWave) == 16 + 64 + 2 * 64 * 8
    assert C.sizeof(capi.TimsField) == C.sizeof(orc.OTims) == 16 + 5 * 8 + 3 * 64 * 8
    waves, tims = time_field_structs(dict(instrument="TIMS", tims=1, tims_z="0,0.01", tims_pi="1,2", tims_pf="3,4",
                                          wave_ramp="0|0|0|0.5"))
    assert tims.n_nodes == 2 and tims.has_final_profile == 1
    assert waves[capi.CHANNEL_TIMS_RAMP_FRACTION].p[0] == 0.5
