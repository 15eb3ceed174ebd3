"""Test helpers: ensemble dictionaries for the golden cases and oracle state
conversion."""
from __future__ import annotations

import json

import numpy as np

from icarion_b200 import _capi as capi
from icarion_b200 import config as cfg
from icarion_b200.sim import IonState

AMU = cfg.AMU_TO_KG
E_CHARGE = cfg.ELEM_CHARGE_C


WAVE_JSON_KEYS = {
    0: ("constant", ["value"]),
    1: ("linear", ["start", "end", "start_time_s", "end_time_s"]),
    2: ("quadratic", ["a", "b", "c", "start_time_s", "end_time_s"]),
    3: ("exponential", ["offset", "amplitude", "rate_per_s", "start_time_s", "end_time_s"]),
    4: ("sinusoidal", ["offset", "amplitude", "frequency_Hz", "phase_rad"]),
    5: ("pwm", ["low", "high", "frequency_Hz", "duty_cycle", "phase_rad", "start_time_s", "end_time_s"]),
    6: ("pulsed", ["low", "high", "pulse_start_s", "pulse_width_s"]),
}


def wave_json(spec: str) -> dict:
    """Harness waveform spec -> the reference's waveform JSON object
    (WaveformLoader.cpp:60-262 field names)."""
    import oracle as orc
    d = orc.parse_wave(spec)
    if d["type"] == 7:
        return {"type": "arbitrary", "times": d["times"], "values": d["values"],
                "interpolation": ("linear", "step", "cubic")[d["interp"]]}
    name, keys = WAVE_JSON_KEYS[d["type"]]
    obj = {"type": name, **{k: d["p"][i] for i, k in enumerate(keys)}}
    if d["type"] in (1, 3, 5):
        obj["clamp"] = bool(d["clamp"])
    return obj


def time_field_structs(kw: dict) -> tuple[dict, object]:
    """Waveform channels and TIMS field of the harness keys as ABI structs,
    every channel evaluated (the reference's waveform_ref semantics)."""
    import oracle as orc
    chans = range(capi.N_CHANNELS)          # the order of orc.WAVE_KEYS
    waves = {ch: orc.wave_struct(kw[key], cls=capi.Waveform) for ch, key in zip(chans, orc.WAVE_KEYS) if key in kw}
    tims = orc.tims_struct(kw, cls=capi.TimsField,
                           names=("initial_uniform_V_m", "final_uniform_V_m", "ramp_start_s", "ramp_end_s",
                                  "ramp_tau_s", "z_positions_m", "initial_profile_V_m", "final_profile_V_m"))
    return waves, tims


def oracle_time_field(kw: dict) -> dict:
    """The harness keys the reference's field model reads: inline waveforms
    of IMS / QuadrupoleRF domains read as 0 V (AnalyticalFieldModel.cpp
    :140-147, 226-233), so those channels are dropped."""
    import oracle as orc
    if kw.get("wave_ref") or kw.get("tims") or kw["instrument"] in ("LQIT", "TIMS"):
        return dict(kw)
    return {k: v for k, v in kw.items() if k not in orc.WAVE_KEYS}


def apply_time_field(sim, kw: dict, ensemble: int = 0) -> None:
    """Waveforms / TIMS field of the harness keys on a Simulation: through
    the JSON adapter (config.time_fields), or as direct structs for
    waveform_ref domains (wave_ref=1), which JSON cannot express."""
    if kw.get("wave_ref"):
        waves, tims = time_field_structs(kw)
    else:
        waves, tims = cfg.time_fields(domain_json(kw))
    if tims is not None:
        sim.set_tims_field(ensemble, tims)
    for ch, w in waves.items():
        sim.set_waveform(ensemble, ch, w)


def domain_json(kw: dict) -> dict:
    """Harness key=value domain (tests/golden/make_golden.py) -> reference JSON domain."""
    dc = {}
    for k1, k2 in (("EN_Td", "EN_Td"), ("axial_V", "axial_V"), ("radial_V", "radial_V"), ("dc_quad_V", "quad_V")):
        if k1 in kw:
            dc[k2] = kw[k1]
    rf = {"voltage_V": kw.get("rf_V", 0.0), "frequency_Hz": kw.get("rf_f", 0.0)}
    for key, blk, name in (("wave_axial", dc, "axial_V"), ("wave_quad", dc, "quad_V"),
                           ("wave_rfv", rf, "voltage_V"), ("wave_rff", rf, "frequency_Hz")):
        if key in kw:
            blk[name] = wave_json(kw[key])
    ac = {"voltage_V": kw.get("ac_V", 0.0), "frequency_Hz": kw.get("ac_f", 0.0), "phase_rad": kw.get("ac_phase", 0.0)}
    dip = {a: {"amplitude_V": kw[f"dip_{a}_A"], "frequency_Hz": kw.get(f"dip_{a}_f", 0.0),
               "phase_rad": kw.get(f"dip_{a}_phase", 0.0), "ramp": kw.get(f"dip_{a}_ramp", 1.0)}
           for a in ("x", "y") if f"dip_{a}_A" in kw}
    if dip:
        ac["dipolar_excitation"] = dip
        for a in ("x", "y"):
            for key, name in ((f"wave_ac{a}A", "amplitude_V"), (f"wave_ac{a}f", "frequency_Hz"),
                              (f"wave_ac{a}r", "ramp")):
                if key in kw and a in dip:
                    dip[a][name] = wave_json(kw[key])
    else:
        for key, name in (("wave_acxA", "voltage_V"), ("wave_acxf", "frequency_Hz")):
            if key in kw:
                ac[name] = wave_json(kw[key])
    return {
        "instrument": kw["instrument"],
        "geometry": {"origin_m": [0.0, 0.0, kw.get("origin_z", 0.0)], "length_m": kw["length"], "radius_m": kw["radius"]},
        "env": {"temperature_K": kw["T"], "pressure_Pa": kw["P"], "gas_species": kw["gas"]},
        "fields": {"DC": dc, "RF": rf, "AC": ac,
                   "magnetic": {"enabled": bool(kw.get("magnetic", 0)), "field_strength_T": [0.0, 0.0, kw.get("B_z", 0.0)]},
                   **({"TIMS": tims_json(kw)} if kw.get("tims") else {})},
    }


def tims_json(kw: dict) -> dict:
    """Harness TIMS keys -> the reference's fields.TIMS block."""
    num = lambda x: [float(v) for v in str(x).split(",") if v != ""]
    t = {"enabled": True, "axial_field_initial_uniform_V_m": float(kw.get("tims_ei", 0.0)),
         "axial_field_final_uniform_V_m": float(kw.get("tims_ef", 0.0)),
         "ramp_start_s": float(kw.get("tims_t0", 0.0)), "ramp_end_s": float(kw.get("tims_t1", 0.0)),
         "ramp_mode": "exponential" if int(kw.get("tims_mode", 0)) else "linear",
         "ramp_tau_s": float(kw.get("tims_tau", 1e-3))}
    if kw.get("tims_z"):
        t["z_positions_m"] = num(kw["tims_z"])
        t["axial_field_initial_profile_V_m"] = num(kw["tims_pi"])
        if kw.get("tims_pf"):
            t["axial_field_final_profile_V_m"] = num(kw["tims_pf"])
    if "wave_ramp" in kw:
        t["ramp_fraction"] = wave_json(kw["wave_ramp"])
    return t


def ensemble_from_golden(z, sigma_m2: float = 150e-20, detector_z_m: float = 1e30) -> dict:
    kw = json.loads(str(z["domain"]))
    dt = float(z["dt"])
    return cfg.ensemble_params(domain_json(kw), sigma_m2, dt, detector_z_m=detector_z_m)


CONFIG0_DOMAIN = {"instrument": "IMS", "origin_z": -0.01, "length": 0.1, "radius": 0.05, "T": 300, "P": 1000,
                  "gas": "N2", "EN_Td": 20}


def config0_ensemble(detector_z_m: float = 2.0e-3, dt: float = 5e-10) -> dict:
    return cfg.ensemble_params(domain_json(CONFIG0_DOMAIN), 150e-20, dt, detector_z_m=detector_z_m)


def golden_state(z, prefix: str = "in_") -> IonState:
    g = {k: np.ascontiguousarray(z[prefix + k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "charge")}
    return IonState(active=np.ascontiguousarray(z[prefix + "active"]).astype(np.uint8),
                    t_death=np.full(g["x"].shape[0], -1.0), t_arrival=np.full(g["x"].shape[0], -1.0), **g)


def oracle_state(st: IonState) -> dict:
    d = {k: np.array(getattr(st, k), dtype=np.float64, copy=True) for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "charge")}
    d["active"] = np.array(st.active, dtype=np.uint8, copy=True)
    d["t_death"] = np.full(st.n, -1.0)
    d["t_arrival"] = np.full(st.n, -1.0)
    return d


def config0_ions(n: int, seed: int = 123):
    """Config-0 cloud: gaussian sigma 0.5 mm at the origin, thermal 300 K, 200 Da, +1."""
    from icarion_b200.sim import generate_ions
    spec = cfg.species_spec(n, 200.0 * AMU, E_CHARGE, {"type": "gaussian", "center": [0, 0, 0], "std": [5e-4] * 3},
                            {"type": "thermal", "temperature_K": 300.0})
    return generate_ions(seed, [spec])


def ion_cloud(n: int, mass_amu: float, seed: int = 123):
    """Seed-123 IonLoader cloud of +1 ions: gaussian sigma 0.5 mm at the
    origin, thermal at 300 K (the reference harness's init mode)."""
    from icarion_b200.sim import generate_ions
    spec = cfg.species_spec(n, mass_amu * AMU, E_CHARGE, {"type": "gaussian", "center": [0, 0, 0], "std": [5e-4] * 3},
                            {"type": "thermal", "temperature_K": 300.0})
    return generate_ions(seed, [spec])


def ipm_reference_case(z):
    """(ensemble, initial ions, fit) of the reference interaction-potential
    fixture ipm_ref_40Td.npz; fit(moments) gives v_drift, K0, D_L, D_T with
    standard errors (icarion_b200.observables)."""
    from icarion_b200 import ipm
    from icarion_b200 import observables as ob
    setup = ipm.IpmSetup()
    dt = float(z["dt"])
    e = cfg.ensemble_params(domain_json(json.loads(str(z["domain"]))), 0.0, dt, detector_z_m=1e30,
                            ipm_bmax_m=setup.b_max_m)
    st0 = ion_cloud(int(z["n_ions"]), float(z["ion_mass_amu"]), int(z["seed"]))
    snap, ref = int(z["snap_every"]), int(z["ref_step"])
    e_z = e["axial_V"] / e["length_m"]

    def fit(mom):
        t = np.arange(1, mom.shape[0] + 1) * snap * dt
        f = ob.fit_transport(t, mom, t_ref=ref * dt)
        f["K0"] = ob.k0_from_drift(f["v_drift"], e_z, e["gas_density_m3"])
        f["se_K0"] = f["K0"] * f["se_v_drift"] / f["v_drift"]
        return f

    return setup, e, st0, fit


def assert_transport_close(got: dict, want: dict, n_sigma: float = 4.0) -> None:
    """v_drift, K0, D_L, D_T within n_sigma combined standard errors."""
    for key in ("v_drift", "K0", "D_L", "D_T"):
        se = float(np.hypot(got["se_" + key], want["se_" + key]))
        assert abs(got[key] - want[key]) <= n_sigma * se, (key, got[key], want[key], se)
