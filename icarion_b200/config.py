"""ICARION JSON config (the unchanged reference schema) -> ensemble parameters.

Only the subset on the uniform-dt batch step is read: ``simulation``
(dt_s, total_time_s, write_interval, integrator, enable_gpu, rng_seed),
``physics.collision_model``, ``domains[]`` (instrument, geometry, env,
fields.DC / RF / magnetic) and ``ions.species[]``.  Derived values are
computed with the reference loader's arithmetic:

* n = P / (kB T)                       EnvironmentConfig.h:152
* axial_V = (E/N [Td] * 1e-21 * n) * L  DomainConfigLoader.cpp:417-431
* mass = mass_amu * AMU_TO_KG, q = charge * e, CCS = CCS_A2 * 1e-20
                                        SpeciesConfig.h:72-84
* gas mass from the species constants  EnvironmentConfig.h:164-200, utils/constants.h

Knobs that are not part of the reference schema (precision mode, steps per
launch, detector plane, ...) are passed separately, never inside the JSON.
"""
from __future__ import annotations

import copy
import json
import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any

from . import _capi as capi

# utils/constants.h
AMU_TO_KG = 1.66053906660e-27
ELEM_CHARGE_C = 1.602176634e-19
BOLTZMANN_CONSTANT = 1.380649e-23
ANGSTROM_TO_M = 1e-10
ANGSTROM2_TO_M2 = 1e-20
ANGSTROM3_TO_M3 = 1e-30
STP_TEMP = 273.15
STP_PRESSURE = 101325.0
EPSILON_0 = 8.854187817e-12

GAS_MASS_KG = {
    "He": 4.002602 * AMU_TO_KG,
    "Ar": 39.948 * AMU_TO_KG,
    "CO2": 44.0095 * AMU_TO_KG,
    "Ne": 20.1797 * AMU_TO_KG,
    "N2": 28.0134 * AMU_TO_KG,
    "O2": 31.9988 * AMU_TO_KG,
    "H2O": 18.01528 * AMU_TO_KG,
}
GAS_POLARIZABILITY_M3 = {
    "He": 0.195e-30, "Ar": 1.596e-30, "CO2": 2.612e-30, "Ne": 0.352e-30,
    "N2": 1.74e-30, "O2": 1.567e-30, "H2O": 1.45e-30,
}

# Every TIMS domain (and every domain with an enabled fields.TIMS block) is
# stepped in TIMSAxialFieldModel (PhysicsSetup.cpp:190-196)
INSTRUMENTS = {"IMS": capi.INSTRUMENT_IMS, "TIMS": capi.INSTRUMENT_TIMS, "FTICR": capi.INSTRUMENT_FTICR,
               "QuadrupoleRF": capi.INSTRUMENT_QUADRUPOLE_RF, "LQIT": capi.INSTRUMENT_LQIT}

WAVE_TYPES = {"constant": capi.WAVE_CONSTANT, "linear": capi.WAVE_LINEAR, "quadratic": capi.WAVE_QUADRATIC,
              "exponential": capi.WAVE_EXPONENTIAL, "sinusoidal": capi.WAVE_SINUSOIDAL, "pwm": capi.WAVE_PWM,
              "pulsed": capi.WAVE_PULSED, "arbitrary": capi.WAVE_ARBITRARY}


def waveform(obj: dict) -> capi.Waveform:
    """A waveform JSON object -> icb_waveform, with WaveformLoader's
    required fields, defaults and checks (WaveformLoader.cpp:60-262)."""
    kind = obj.get("type")
    if kind not in WAVE_TYPES:
        raise ValueError(f"unknown waveform type {kind!r}")
    w = capi.Waveform()
    w.type = WAVE_TYPES[kind]
    if kind in ("linear", "exponential", "pwm"):
        w.clamp = int(bool(obj.get("clamp", True)))
    req = lambda k: float(obj[k])
    opt = lambda k, d: float(obj.get(k, d))
    if kind == "constant":
        p = [req("value")]
    elif kind == "linear":
        p = [req("start"), req("end"), opt("start_time_s", 0.0), req("end_time_s")]
        if p[3] <= p[2]:
            raise ValueError("LinearWaveform: end_time_s must be > start_time_s")
    elif kind == "quadratic":
        p = [req("a"), req("b"), req("c"), opt("start_time_s", 0.0), opt("end_time_s", 1e9)]
    elif kind == "exponential":
        p = [opt("offset", 0.0), req("amplitude"), req("rate_per_s"), opt("start_time_s", 0.0), opt("end_time_s", 1e9)]
        if p[4] <= p[3]:
            raise ValueError("ExponentialWaveform: end_time_s must be > start_time_s")
    elif kind == "sinusoidal":
        p = [opt("offset", 0.0), req("amplitude"), req("frequency_Hz"), opt("phase_rad", 0.0)]
        if p[2] <= 0.0:
            raise ValueError("SinusoidalWaveform: frequency_Hz must be positive")
    elif kind == "pwm":
        p = [req("low"), req("high"), req("frequency_Hz"), req("duty_cycle"), opt("phase_rad", 0.0),
             opt("start_time_s", 0.0), opt("end_time_s", 1e9)]
        if p[2] <= 0.0 or not 0.0 <= p[3] <= 1.0 or p[6] <= p[5]:
            raise ValueError("PWMWaveform: needs frequency > 0, duty_cycle in [0, 1], end_time_s > start_time_s")
    elif kind == "pulsed":
        p = [req("low"), req("high"), req("pulse_start_s"), req("pulse_width_s")]
        if p[3] <= 0.0 or p[2] < 0.0:
            raise ValueError("PulsedWaveform: needs pulse_width_s > 0 and pulse_start_s >= 0")
    else:
        times = [float(v) for v in obj["times"]]
        values = [float(v) for v in obj["values"]]
        if len(times) != len(values) or len(times) < 2:
            raise ValueError("ArbitraryWaveform: 'times' and 'values' need the same length >= 2")
        if any(b <= a for a, b in zip(times, times[1:])):
            raise ValueError("ArbitraryWaveform: times must be strictly increasing")
        if len(times) > capi.MAX_WAVE_POINTS:
            raise ValueError(f"ArbitraryWaveform: at most {capi.MAX_WAVE_POINTS} points")
        w.interp = {"linear": capi.INTERP_LINEAR, "step": capi.INTERP_STEP,
                    "cubic": capi.INTERP_CUBIC}[obj.get("interpolation", "linear")]
        w.n_points = len(times)
        w.times_s[:len(times)] = times
        w.values[:len(values)] = values
        p = []
    w.p[:] = (p + [0.0] * 8)[:8]
    return w


def value_or_waveform(v: Any, library: dict) -> float | capi.Waveform:
    """ValueOrWaveform JSON (number, "@id" or inline object) -> a constant or
    a waveform (WaveformLoader::load_value_or_waveform; "@id" resolves to an
    inline copy, local library first)."""
    if isinstance(v, (int, float)):
        return float(v)
    if isinstance(v, str):
        if not v.startswith("@"):
            raise ValueError(f"waveform reference must start with '@' (got {v!r})")
        if v[1:] not in library:
            raise ValueError(f"waveform reference not found: {v[1:]}")
        return waveform(library[v[1:]])
    return waveform(v)


def wave_value(w: capi.Waveform, t: float) -> float:
    """A waveform's value at one time t (host; the FTICR radial voltage is
    read once at t = 0, AnalyticalFieldModel.cpp:174-176)."""
    p = list(w.p)
    if w.type == capi.WAVE_CONSTANT:
        return p[0]
    if w.type == capi.WAVE_LINEAR:
        if t < p[2]:
            return p[0]
        if t >= p[3]:
            return p[1] if w.clamp else p[0]
        return p[0] + (p[1] - p[0]) * ((t - p[2]) / (p[3] - p[2]))
    if w.type == capi.WAVE_QUADRATIC:
        return p[0] if (t < p[3] or t > p[4]) else p[0] + p[1] * t + p[2] * t * t
    if w.type == capi.WAVE_EXPONENTIAL:
        rel = 0.0 if t < p[3] else ((p[4] - p[3]) if w.clamp else 0.0) if t >= p[4] else t - p[3]
        return p[0] + p[1] * math.exp(p[2] * rel)
    if w.type == capi.WAVE_SINUSOIDAL:
        return p[0] + p[1] * math.sin(2.0 * math.pi * p[2] * t + p[3])
    if w.type == capi.WAVE_PWM:
        if p[2] <= 0.0 or t < p[5] or (t >= p[6] and not w.clamp):
            return p[0]
        tr = (p[6] - p[5]) if t >= p[6] else t - p[5]
        period = 1.0 / p[2]
        ph = math.fmod(tr + p[4] / (2.0 * math.pi * p[2]), period)
        ph = ph + period if ph < 0.0 else ph
        return p[1] if ph < p[3] * period else p[0]
    if w.type == capi.WAVE_PULSED:
        return p[1] if p[2] <= t < p[2] + p[3] else p[0]
    n = w.n_points
    ts, vs = list(w.times_s[:n]), list(w.values[:n])
    if t <= ts[0]:
        return vs[0]
    if t >= ts[-1]:
        return vs[-1]
    i1 = next(i for i, x in enumerate(ts) if x >= t)
    i0 = i1 - 1
    if w.interp == capi.INTERP_STEP:
        return vs[i0]
    a = (t - ts[i0]) / (ts[i1] - ts[i0])
    if w.interp == capi.INTERP_LINEAR:
        return vs[i0] + a * (vs[i1] - vs[i0])
    raise ValueError("cubic interpolation is evaluated on the device only")


def _scalar(v: Any) -> float:
    """The constant of a ValueOrWaveform slot; 0 for a waveform (carried by
    time_fields)."""
    return float(v) if isinstance(v, (int, float)) else 0.0


def _tims_block(fields: dict) -> dict | None:
    t = fields.get("TIMS", fields.get("tims"))
    if t is None or not t.get("enabled", True):
        return None
    return t


def uses_tims_model(domain: dict) -> bool:
    """PhysicsSetup.cpp:190-196: instrument TIMS or fields.TIMS.enabled."""
    return domain.get("instrument", "IMS") == "TIMS" or _tims_block(domain.get("fields", {})) is not None


def time_fields(domain: dict, global_waveforms: dict | None = None) -> tuple[dict, capi.TimsField | None]:
    """Waveform channels and TIMS axial field of one domain, as the
    reference's field model evaluates them: {ICB_CHANNEL_*: icb_waveform}
    and an icb_tims_field (or None).

    IMS and QuadrupoleRF read a voltage only when it is a constant or a
    waveform_ref (AnalyticalFieldModel.cpp:140-147, 226-233), and the loader
    turns every waveform, "@id" included, into an inline copy
    (WaveformLoader.cpp:290-320): their waveforms read as 0 V.  The LQIT
    and TIMS models evaluate inline waveforms (:41-45, TIMSAxialFieldModel.h
    :60-64)."""
    fields = domain.get("fields", {})
    lib = dict(global_waveforms or {})
    lib.update(fields.get("waveforms", {}) or {})
    dc = fields.get("DC", fields.get("dc", {})) or {}
    rf = fields.get("RF", fields.get("rf", {})) or {}
    tims_on = uses_tims_model(domain)
    inst = domain.get("instrument", "IMS")
    evaluates_inline = tims_on or inst == "LQIT"
    waves = {}
    slots = ((capi.CHANNEL_DC_AXIAL_V, dc, "axial_V"), (capi.CHANNEL_DC_QUAD_V, dc, "quad_V"),
             (capi.CHANNEL_RF_VOLTAGE_V, rf, "voltage_V"), (capi.CHANNEL_RF_FREQUENCY_HZ, rf, "frequency_Hz"))
    for ch, blk, key in slots:
        if key not in blk or not evaluates_inline:
            continue
        v = value_or_waveform(blk[key], lib)
        if isinstance(v, capi.Waveform):
            waves[ch] = v
    if inst == "LQIT" and not tims_on:
        dip, ac_slots = _ac_slots(fields)
        for a, sl in enumerate(ac_slots):
            if sl is None:
                continue
            base = capi.CHANNEL_AC_X_AMPLITUDE_V + 3 * a
            for j, v in enumerate(sl[:3] if dip else sl[:2]):
                v = value_or_waveform(v, lib)
                if isinstance(v, capi.Waveform):
                    waves[base + j] = v
    tims = None
    # the TIMS model reads the block's values whether or not it is enabled
    tb = fields.get("TIMS", fields.get("tims"))
    if tims_on and tb is not None:
        tims = capi.TimsField()
        mode = tb.get("ramp_mode", "linear")
        if mode not in ("linear", "exponential"):
            raise ValueError("TIMS ramp_mode must be 'linear' or 'exponential'")
        tims.ramp_mode = capi.TIMS_RAMP_EXPONENTIAL if mode == "exponential" else capi.TIMS_RAMP_LINEAR
        tims.initial_uniform_V_m = float(tb.get("axial_field_initial_uniform_V_m", 0.0))
        tims.final_uniform_V_m = float(tb.get("axial_field_final_uniform_V_m", 0.0))
        tims.ramp_start_s = float(tb.get("ramp_start_s", 0.0))
        tims.ramp_end_s = float(tb.get("ramp_end_s", 0.0))
        tims.ramp_tau_s = float(tb.get("ramp_tau_s", 1e-3))
        z = [float(v) for v in tb.get("z_positions_m", [])]
        pi = [float(v) for v in tb.get("axial_field_initial_profile_V_m", [])]
        pf = [float(v) for v in tb.get("axial_field_final_profile_V_m", [])]
        if z:
            if len(z) < 2 or len(pi) != len(z) or (pf and len(pf) != len(z)):
                raise ValueError("TIMS profiles need >= 2 z positions and matching profile sizes")
            if len(z) > capi.MAX_WAVE_POINTS:
                raise ValueError(f"TIMS profiles take at most {capi.MAX_WAVE_POINTS} nodes")
            tims.n_nodes = len(z)
            tims.has_final_profile = int(bool(pf))
            tims.z_positions_m[:len(z)] = z
            tims.initial_profile_V_m[:len(pi)] = pi
            tims.final_profile_V_m[:len(pf)] = pf
        if "ramp_fraction" in tb:
            v = value_or_waveform(tb["ramp_fraction"], lib)
            if not isinstance(v, capi.Waveform):
                c = capi.Waveform()
                c.type = capi.WAVE_CONSTANT
                c.p[0] = v
                v = c
            waves[capi.CHANNEL_TIMS_RAMP_FRACTION] = v
    return waves, tims


def ac_drives(fields: dict) -> tuple[list[float], list[float], list[float], list[float], int]:
    """fields.AC of an LQIT (DomainConfigLoader.cpp:262-275, 505-545;
    FieldsConfig.h:93-168) -> per-axis (amplitude V, frequency Hz, phase rad)
    and ramp for x and y, and whether the drive is the two-axis dipolar one
    (AC.dipolar_excitation, the AC.x / AC.y shorthand or
    fields.dipolar_excitation; a disabled axis gets amplitude 0); otherwise
    the single-axis AC.voltage_V drives x.  Constant values only."""
    dip, slots = _ac_slots(fields)
    amp, freq, phase, ramp = [0.0, 0.0], [0.0, 0.0], [0.0, 0.0], [1.0, 1.0]
    for a, sl in enumerate(slots):
        if sl is None:
            continue
        amp[a], freq[a], phase[a] = _scalar(sl[0]), _scalar(sl[1]), float(sl[3])
        ramp[a] = _scalar(sl[2]) if dip else 1.0
    return amp, freq, phase, ramp, int(dip)


def _ac_slots(fields: dict) -> tuple[bool, list]:
    """The AC drive's (amplitude, frequency, ramp, phase) JSON values per
    axis (None for an absent or disabled axis) and whether the drive is the
    two-axis dipolar one."""
    ac = fields.get("AC", fields.get("ac", {})) or {}
    dip = fields.get("dipolar_excitation")
    if dip is None:
        dip = ac.get("dipolar_excitation")
    if dip is None and ("x" in ac or "y" in ac):
        dip = {k: ac[k] for k in ("x", "y") if k in ac}
    if dip is None:
        return False, [(ac.get("voltage_V", 0.0), ac.get("frequency_Hz", 0.0), 1.0, ac.get("phase_rad", 0.0)), None]
    slots = []
    for key in ("x", "y"):
        axis = dip.get(key)
        if not axis or not axis.get("enabled", True):
            slots.append(None)
            continue
        slots.append((axis.get("amplitude_V", axis.get("voltage_V", 0.0)), axis.get("frequency_Hz", 0.0),
                      axis.get("ramp", 1.0), axis.get("phase_rad", 0.0)))
    return True, slots
INTEGRATORS = {"Boris": capi.INTEGRATOR_BORIS, "RK4": capi.INTEGRATOR_RK4}
COLLISIONS = {"None": capi.COLLISION_NONE, "none": capi.COLLISION_NONE, "HSS": capi.COLLISION_HSS,
              "IPM": capi.COLLISION_IPM_TABLE}


def gas_density(pressure_pa: float, temperature_k: float) -> float:
    """n = P / (kB T) (EnvironmentConfig::compute_derived_properties)."""
    return pressure_pa / (BOLTZMANN_CONSTANT * temperature_k)


def axial_voltage_from_en(en_td: float, pressure_pa: float, temperature_k: float, length_m: float) -> float:
    """E/N [Td] -> axial_V exactly as DomainConfigLoader::load_dc_fields."""
    k_b = 1.380649e-23
    n = pressure_pa / (k_b * temperature_k)
    e_vm = en_td * 1e-21 * n
    return e_vm * length_m


def thermal_width(temperature_k: float, mass_kg: float) -> float:
    return math.sqrt(BOLTZMANN_CONSTANT * temperature_k / mass_kg)


def n0_loschmidt() -> float:
    """N0 = 101325 / (kB * 273.15) used to reduce mobilities to K0."""
    return STP_PRESSURE / (BOLTZMANN_CONSTANT * STP_TEMP)


@dataclass
class Species:
    species_id: str
    mass_kg: float
    charge_C: float
    ccs_m2: float
    ccs_hss_m2: dict = field(default_factory=dict)

    def sigma_for_gas(self, gas: str) -> float:
        return self.ccs_hss_m2.get(gas, self.ccs_m2)


def species_from_db_entry(sid: str, e: dict) -> Species:
    ccs = e.get("CCS_A2")
    return Species(
        species_id=sid,
        mass_kg=float(e["mass_amu"]) * AMU_TO_KG,
        charge_C=int(e["charge"]) * ELEM_CHARGE_C,
        ccs_m2=(float(ccs) * ANGSTROM2_TO_M2) if ccs is not None else 0.0,
        ccs_hss_m2={g: float(v) * ANGSTROM2_TO_M2 for g, v in e.get("CCS_HSS", {}).items()},
    )


def ensemble_params(domain: dict, sigma_m2: float, dt_s: float, detector_z_m: float = 1e30,
                    ipm_bmax_m: float = 0.0, sigma_by_gas: dict | None = None) -> dict:
    """One ensemble (domain + env + ion cross-section + dt) as a plain dict.

    ``env.gas_mixture`` (a list of {species, mole_fraction[, cross_section_m2]})
    becomes the HSS mixture: densities f_i P/(kB T) with the fractions
    normalised as EnvironmentConfig::compute_derived_properties does
    (EnvironmentConfig.h:155-170), cross-sections from the component's
    override, else ``sigma_by_gas[species]``, else ``sigma_m2``
    (HSSCollisionHandler.cpp:136-176)."""
    geom = domain.get("geometry", {})
    env = domain.get("env", domain.get("environment", {}))
    fields = domain.get("fields", {})
    dc = fields.get("DC", fields.get("dc", {}))
    rf = fields.get("RF", fields.get("rf", {}))
    mag = fields.get("magnetic", {})
    T = float(env.get("temperature_K", 300.0))
    P = float(env.get("pressure_Pa", 101325.0))
    gas = env.get("gas_species", "He")
    L = float(geom.get("length_m", 0.1))
    mix = env.get("gas_mixture", []) or []
    # densities from the normalised mole fractions of all components
    # (EnvironmentConfig.h:155-175); only those that take part in collisions
    # enter the collision law (HSSCollisionHandler.cpp:127-133)
    fsum = sum(float(c.get("mole_fraction", 0.0)) for c in mix)
    norm = fsum if fsum > 0.0 else 1.0
    n_tot = gas_density(P, T)
    comps = []
    for c in mix:
        n_i = float(c.get("mole_fraction", 0.0)) / norm * n_tot
        if not c.get("participates_in_collisions", True) or n_i <= 0.0:
            continue
        override = float(c.get("cross_section_m2", -1.0))
        comps.append((n_i, GAS_MASS_KG.get(c["species"], GAS_MASS_KG["He"]),
                      override if override > 0.0 else float((sigma_by_gas or {}).get(c["species"], sigma_m2))))
    if len(comps) > 8:
        raise ValueError("at most 8 gas mixture components")
    n_mix = len(comps) if len(comps) >= 2 else 0
    dens, mass, sig = [0.0] * 8, [0.0] * 8, [0.0] * 8
    for i, (n_i, m_i, s_i) in enumerate(comps if n_mix else []):
        dens[i], mass[i], sig[i] = n_i, m_i, s_i
    # a mixture with one colliding component is that component alone; with
    # none, no collisions
    single_gas = (gas_density(P, T), GAS_MASS_KG[gas], float(sigma_m2))
    if mix and len(comps) == 1:
        single_gas = comps[0]
    elif mix and not comps:
        single_gas = (0.0, GAS_MASS_KG[gas], float(sigma_m2))
    ac_amp, ac_freq, ac_phase, ac_ramp, ac_dipolar = ac_drives(fields)
    axial = 0.0
    if isinstance(dc.get("EN_Td"), (int, float)):
        axial = axial_voltage_from_en(float(dc["EN_Td"]), P, T, L)
    if "axial_V" in dc:
        axial = _scalar(dc["axial_V"])
    radial = dc.get("radial_V", 0.0)
    if not isinstance(radial, (int, float)):
        lib = fields.get("waveforms", {}) or {}
        radial = wave_value(value_or_waveform(radial, lib), 0.0)
    instrument = INSTRUMENTS[domain.get("instrument", "IMS")]
    if uses_tims_model(domain):
        instrument = capi.INSTRUMENT_TIMS
    return {
        "instrument": instrument,
        "magnetic_enabled": int(bool(mag.get("enabled", False))),
        "origin_m": [float(v) for v in geom.get("origin_m", [0.0, 0.0, 0.0])],
        "length_m": L,
        "radius_m": float(geom.get("radius_m", 0.05)),
        "axial_V": axial,
        "radial_V": float(radial),
        "dc_quad_V": _scalar(dc.get("quad_V", 0.0)),
        "rf_voltage_V": _scalar(rf.get("voltage_V", 0.0)),
        "rf_frequency_Hz": _scalar(rf.get("frequency_Hz", 0.0)),
        "B_T": [float(v) for v in mag.get("field_strength_T", [0.0, 0.0, 0.0])],
        "temperature_K": T,
        "gas_density_m3": single_gas[0],
        "gas_mass_kg": single_gas[1],
        "gas_velocity_m_s": [float(v) for v in env.get("gas_velocity_m_s", [0.0, 0.0, 0.0])],
        "gas_polarizability_m3": GAS_POLARIZABILITY_M3.get(gas, 0.0),
        "sigma_m2": single_gas[2],
        "ipm_bmax_m": float(ipm_bmax_m),
        "dt_s": float(dt_s),
        "detector_z_m": float(detector_z_m),
        "n_gas": n_mix,
        "flow_model": flow_model(env.get("flow_model", "constant")),
        "gas_mix_density_m3": dens,
        "gas_mix_mass_kg": mass,
        "gas_mix_sigma_m2": sig,
        "axial_flow_velocity_m_s": float(env.get("axial_flow_velocity_m_s", 0.0)),
        "axial_flow_max_velocity_m_s": float(env.get("axial_flow_max_velocity_m_s", 0.0)),
        "ac_amplitude_V": ac_amp,
        "ac_frequency_Hz": ac_freq,
        "ac_phase_rad": ac_phase,
        "ac_ramp": ac_ramp,
        "ac_dipolar": ac_dipolar,
        "reserved2_": 0,
    }


def flow_model(name: str) -> int:
    """env.flow_model names (EnvironmentConfig::parse_flow_model,
    EnvironmentConfig.h:81-94) -> ICB_FLOW_*."""
    key = str(name).lower()
    if key in ("constant", "legacy"):
        return capi.FLOW_CONSTANT
    if key in ("axial_uniform", "uniform", "axial_const"):
        return capi.FLOW_AXIAL_UNIFORM
    if key in ("axial_parabolic", "parabolic", "poiseuille"):
        return capi.FLOW_AXIAL_PARABOLIC
    raise ValueError(f"unknown flow_model '{name}'")


def to_struct(p: dict) -> capi.EnsembleParams:
    s = capi.EnsembleParams()
    for k, _ in capi.EnsembleParams._fields_:
        v = p[k]
        if isinstance(v, (list, tuple)):
            getattr(s, k)[:] = [float(x) for x in v]
        else:
            setattr(s, k, v)
    return s


def species_spec(count: int, mass_kg: float, charge_C: float, position: dict, velocity: dict) -> capi.SpeciesSpec:
    """IonSpeciesConfig position/velocity blocks -> icb_species_spec."""
    s = capi.SpeciesSpec()
    s.count = int(count)
    s.mass_kg = mass_kg
    s.charge_C = charge_C
    ptype = position.get("type", "point").lower()
    s.position_type = {"point": capi.POS_POINT, "gaussian": capi.POS_GAUSSIAN,
                       "uniform_sphere": capi.POS_UNIFORM_SPHERE, "uniform_cylinder": capi.POS_UNIFORM_CYLINDER,
                       "uniform_box": capi.POS_UNIFORM_BOX}[ptype]
    s.center_m[:] = [float(v) for v in position.get("center", [0.0, 0.0, 0.0])]
    s.std_m[:] = [float(v) for v in position.get("std", [0.0, 0.0, 0.0])]
    s.radius_m = float(position.get("radius", 0.0))
    s.length_m = float(position.get("length", 0.0))
    s.box_min_m[:] = [float(v) for v in position.get("min", [0.0, 0.0, 0.0])]
    s.box_max_m[:] = [float(v) for v in position.get("max", [0.0, 0.0, 0.0])]
    vtype = velocity.get("type", "fixed").lower()
    s.velocity_type = {"fixed": capi.VEL_FIXED, "thermal": capi.VEL_THERMAL}[vtype]
    s.velocity_m_s[:] = [float(v) for v in velocity.get("value", [0.0, 0.0, 0.0])]
    s.temperature_K = float(velocity.get("temperature_K", 300.0))
    return s


@dataclass
class RunConfig:
    """The parts of a reference config the batch step needs."""
    dt_s: float
    total_time_s: float
    write_interval: int
    integrator: int
    collision_model: int
    rng_seed: int
    enable_gpu: bool
    domain: dict
    species: list            # list[(Species, count, position, velocity)]
    raw: dict

    @property
    def n_steps(self) -> int:
        return int(round(self.total_time_s / self.dt_s))


def load(cfg: Any, species_db: dict | None = None) -> RunConfig:
    """Read a reference config (path or dict).  ``species_db`` is the parsed
    species database (``{"species": {...}}``); inline entries in it override
    the file named by the config's ``species_database``."""
    if isinstance(cfg, (str, Path)):
        path = Path(cfg)
        raw = json.loads(path.read_text())
        base = path.parent
    else:
        raw = copy.deepcopy(cfg)
        base = Path(".")
    db = {}
    if "species_database" in raw and species_db is None:
        dbp = base / raw["species_database"]
        if dbp.exists():
            db = json.loads(dbp.read_text()).get("species", {})
    if species_db:
        db.update(species_db.get("species", species_db))
    sim = raw["simulation"]
    phys = raw.get("physics", {})
    species = []
    for sp in raw.get("ions", {}).get("species", []):
        spc = species_from_db_entry(sp["id"], db[sp["id"]])
        species.append((spc, int(sp["count"]), sp.get("position", {}), sp.get("velocity", {})))
    return RunConfig(
        dt_s=float(sim["dt_s"]),
        total_time_s=float(sim["total_time_s"]),
        write_interval=int(sim.get("write_interval", 1000)),
        integrator=INTEGRATORS[sim.get("integrator", "RK4")],
        collision_model=COLLISIONS[phys.get("collision_model", "None")],
        rng_seed=int(sim.get("rng_seed", 0)),
        enable_gpu=bool(sim.get("enable_gpu", False)),
        domain=raw["domains"][0],
        species=species,
        raw=raw,
    )
