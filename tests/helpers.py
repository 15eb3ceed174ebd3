"""Test helpers: ensemble dictionaries for the golden cases and oracle state
conversion."""
from __future__ import annotations

import json

import numpy as np

from icarion_b200 import config as cfg
from icarion_b200.sim import IonState

AMU = cfg.AMU_TO_KG
E_CHARGE = cfg.ELEM_CHARGE_C


def domain_json(kw: dict) -> dict:
    """Harness key=value domain (tests/golden/make_golden.py) -> reference JSON domain."""
    dc = {}
    for k1, k2 in (("EN_Td", "EN_Td"), ("axial_V", "axial_V"), ("radial_V", "radial_V"), ("dc_quad_V", "quad_V")):
        if k1 in kw:
            dc[k2] = kw[k1]
    ac = {"voltage_V": kw.get("ac_V", 0.0), "frequency_Hz": kw.get("ac_f", 0.0), "phase_rad": kw.get("ac_phase", 0.0)}
    dip = {a: {"amplitude_V": kw[f"dip_{a}_A"], "frequency_Hz": kw.get(f"dip_{a}_f", 0.0),
               "phase_rad": kw.get(f"dip_{a}_phase", 0.0), "ramp": kw.get(f"dip_{a}_ramp", 1.0)}
           for a in ("x", "y") if f"dip_{a}_A" in kw}
    if dip:
        ac["dipolar_excitation"] = dip
    return {
        "instrument": kw["instrument"],
        "geometry": {"origin_m": [0.0, 0.0, kw.get("origin_z", 0.0)], "length_m": kw["length"], "radius_m": kw["radius"]},
        "env": {"temperature_K": kw["T"], "pressure_Pa": kw["P"], "gas_species": kw["gas"]},
        "fields": {"DC": dc, "RF": {"voltage_V": kw.get("rf_V", 0.0), "frequency_Hz": kw.get("rf_f", 0.0)}, "AC": ac,
                   "magnetic": {"enabled": bool(kw.get("magnetic", 0)), "field_strength_T": [0.0, 0.0, kw.get("B_z", 0.0)]}},
    }


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
