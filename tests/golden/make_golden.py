"""Generate the golden fixtures of tests/golden/ from the reference's own code.

    make -C oracle REF=<reference tree> && python tests/golden/make_golden.py [--quick]

Every fixture is produced by ``oracle/_ref/ref_harness`` — the reference's
hot-path sources (BorisStrategy, RK4Strategy, HSSCollisionHandler,
CollisionKernels, VelocitySampling, PhysicsRng, ForceRegistry, the analytic
field model and CylindricalGeometry) compiled unchanged by oracle/Makefile —
driven through the reference engine's per-step order.  The reference tree is
needed only here; the fixtures travel with the repository.

Fixtures
  rng_mt64.npz          PhysicsRng(seed).uniform01() streams (seeds 123, 4219)
  ions_init.npz         IonLoader gaussian/thermal cloud from std::mt19937(123)
  derived.json          loader-derived n, gas mass, axial_V, E_z (config 0)
  push_<case>.npz       collision-free Boris / RK4 runs (IMS, FTICR, QuadrupoleRF, LQIT)
  hss_ref.npz           Boris + reference HSS, 64 ions x 2000 steps
  ims_config0.npz       config-0 physics: 65,536 ions x 100k steps, moments
                        every 1000 steps, displacement reference after 20k
                        steps, arrival (z = 2 mm) and death times, OpenMP
                        timing (--config0-only regenerates just this one)
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as orc  # noqa: E402

OUT = Path(__file__).resolve().parent
CONFIG0_IONS = 65536
AMU = 1.66053906660e-27
E = 1.602176634e-19

# config 0: IMS drift of 200 Da, 150 A^2 ions in N2, 300 K, 1000 Pa, 20 Td
IMS_DOMAIN = dict(instrument="IMS", origin_z=-0.01, length=0.1, radius=0.05, T=300, P=1000, gas="N2", EN_Td=20)
FTICR_DOMAIN = dict(instrument="FTICR", origin_z=0.0, length=0.05, radius=0.025, T=300, P=1e-7, gas="He",
                    radial_V=1.0, magnetic=1, B_z=7.0)
QUAD_DOMAIN = dict(instrument="QuadrupoleRF", origin_z=-0.05, length=0.1, radius=0.005, T=300, P=1.0, gas="He",
                   rf_V=200.0, rf_f=1.0e6, dc_quad_V=5.0, axial_V=1.0)
# linear ion trap: RF 200 V at 1 MHz (q ~ 0.6 at 200 Da), 2 V axial well,
# two-axis dipolar drive (single-axis drive in LQIT1_DOMAIN)
LQIT_DOMAIN = dict(instrument="LQIT", origin_z=-0.025, length=0.05, radius=0.004, T=300, P=0.1, gas="He",
                   rf_V=200.0, rf_f=1.0e6, dc_quad_V=1.0, axial_V=2.0,
                   dip_x_A=0.5, dip_x_f=1.0e5, dip_x_phase=0.3, dip_x_ramp=0.8, dip_y_A=0.2, dip_y_f=1.2e5)
LQIT1_DOMAIN = dict(instrument="LQIT", origin_z=-0.025, length=0.05, radius=0.004, T=300, P=0.1, gas="He",
                    rf_V=200.0, rf_f=1.0e6, axial_V=2.0, ac_V=0.4, ac_f=9.0e4, ac_phase=1.1)


# Time-dependent fields.  Waveform specs are "type|clamp|interp|params|times|values"
# with the types in WaveformType order (constant, linear, quadratic,
# exponential, sinusoidal, pwm, pulsed, arbitrary).
# TIMS (TIMSAxialFieldModel): profile ramp over 1..4 us, RF confinement
TIMS_DOMAIN = dict(instrument="TIMS", origin_z=-0.01, length=0.02, radius=0.005, T=300, P=310.0, gas="N2",
                   rf_V=180.0, rf_f=2.0e6, dc_quad_V=0.0, tims=1, tims_z="0,0.02", tims_pi="0,-449.5",
                   tims_pf="0,0", tims_t0=1e-6, tims_t1=4e-6)
# exponential ramp between uniform fields, DC quadrupole offset
TIMS_EXP_DOMAIN = dict(instrument="TIMS", origin_z=-0.01, length=0.02, radius=0.005, T=300, P=310.0, gas="N2",
                       rf_V=150.0, rf_f=1.5e6, dc_quad_V=2.0, tims=1, tims_mode=1, tims_ei=-300.0, tims_ef=-100.0,
                       tims_t0=5e-7, tims_t1=3.5e-6, tims_tau=1e-6)
# an enabled TIMS block on an IMS domain: ramp fraction from a cubic
# arbitrary waveform (clamped above 1), three-node initial profile, final
# uniform field, RF frequency ramp
TIMS_WAVE_DOMAIN = dict(instrument="IMS", origin_z=-0.01, length=0.02, radius=0.005, T=300, P=310.0, gas="N2",
                        rf_V=180.0, rf_f=2.0e6, tims=1, tims_z="0,0.008,0.02", tims_pi="-100,-400,-250",
                        tims_ef=-50.0, wave_ramp="7|0|2||0,1e-6,2e-6,3e-6,4e-6|0,0.1,0.5,0.9,1.2",
                        wave_rff="1|1|0|2e6,2.2e6,0,4e-6")
# LQIT with an axial ramp, modulated RF amplitude, chirped RF frequency and
# a gated PWM DC quadrupole
LQIT_WAVE_DOMAIN = dict(LQIT_DOMAIN, wave_axial="1|1|0|2,5,0,4e-6", wave_rfv="4|0|0|200,20,2e5,0.3",
                        wave_rff="2|0|0|1e6,1e10,0,0,1e-5", wave_quad="5|0|0|0.5,1.5,5e5,0.3,0.2,1e-6,4e-6")
# LQIT AC drives as waveforms: a resonance scan (chirped x drive faded in,
# pulsed y drive) on the dipolar trap, and a modulated single-axis drive
# with a quadratic chirp
LQIT_AC_DOMAIN = dict(LQIT_DOMAIN, wave_acxf="1|1|0|1e5,2e5,0,4e-6", wave_acxr="1|1|0|0,1,0,2e-6",
                      wave_acyA="6|0|0|0,0.4,1e-6,2e-6")
LQIT1_AC_DOMAIN = dict(LQIT1_DOMAIN, wave_acxA="4|0|0|0.4,0.2,3e5,0", wave_acxf="2|0|0|9e4,2e10,0,0,1e-5")
# IMS / QuadrupoleRF read waveforms given as waveform_ref
IMS_REF_DOMAIN = dict(IMS_DOMAIN, wave_ref=1, wave_axial="3|1|0|1000,500,-3e5,1e-6,6e-6",
                      wave_rfv="6|0|0|0,50,1e-6,2e-6", wave_rff="0|0|0|1e6", wave_quad="7|0|1||0,2e-6,4e-6|0,1,-1")
QUAD_REF_DOMAIN = dict(QUAD_DOMAIN, wave_ref=1, wave_rfv="1|1|0|200,250,0,3e-6", wave_axial="4|0|0|1,0.5,3e5,0")
# ... and read inline waveforms (what the loader makes of "@id" and objects) as 0 V
IMS_INLINE_DOMAIN = dict(IMS_DOMAIN, wave_axial="1|1|0|0,2000,0,2e-6")
# every waveform type, clamp and interpolation on the RF voltage of a
# QuadrupoleRF domain (waveform_ref)
WAVE_TYPE_SPECS = {
    "constant": "0|0|0|190",
    "linear_clamp": "1|1|0|150,250,1e-6,3e-6",
    "linear_hold_start": "1|0|0|150,250,1e-6,3e-6",
    "quadratic": "2|0|0|100,3e7,4e12,5e-7,4e-6",
    "exponential_clamp": "3|1|0|120,80,-6e5,1e-6,4e-6",
    "exponential_noclamp": "3|0|0|120,80,4e5,1e-6,4e-6",
    "sinusoidal": "4|0|0|200,30,7e5,0.4",
    "pwm_clamp": "5|1|0|100,220,8e5,0.35,0.7,5e-7,4.1e-6",
    "pwm_noclamp": "5|0|0|100,220,8e5,0.35,-0.5,5e-7,4.1e-6",
    "pulsed": "6|0|0|80,240,1.5e-6,1e-6",
    "arbitrary_linear": "7|0|0||0,1e-6,2.5e-6,4e-6|100,260,180,220",
    "arbitrary_step": "7|0|1||0,1e-6,2.5e-6,4e-6|100,260,180,220",
    "arbitrary_cubic": "7|0|2||0,1e-6,2.5e-6,4e-6,5e-6|100,260,180,220,150",
}


def field_cases() -> dict:
    cases = {"tims": TIMS_DOMAIN, "tims_exp": TIMS_EXP_DOMAIN, "tims_wave": TIMS_WAVE_DOMAIN,
             "lqit_wave": LQIT_WAVE_DOMAIN, "ims_ref": IMS_REF_DOMAIN, "quadrf_ref": QUAD_REF_DOMAIN,
             "ims_inline": IMS_INLINE_DOMAIN, "lqit_ac": LQIT_AC_DOMAIN, "lqit1_ac": LQIT1_AC_DOMAIN}
    for name, spec in WAVE_TYPE_SPECS.items():
        cases[f"wave_{name}"] = dict(QUAD_DOMAIN, wave_ref=1, wave_rfv=spec)
    return cases


def field_points(kw: dict, n: int = 40, seed: int = 7) -> np.ndarray:
    """(x, y, z, t) rows inside and just outside the cylinder, at times on a
    grid over -1..8 us plus every boundary time the cases use."""
    rng = np.random.default_rng(seed)
    L, R, oz = float(kw["length"]), float(kw["radius"]), float(kw.get("origin_z", 0.0))
    t_edges = [0.0, 5e-7, 1e-6, 1.5e-6, 2e-6, 2.5e-6, 3e-6, 3.5e-6, 4e-6, 4.1e-6, 5e-6, 6e-6]
    t = np.concatenate([np.linspace(-1e-6, 8e-6, n), t_edges])
    m = t.size
    r = R * np.sqrt(rng.random(m))
    ph = 2 * np.pi * rng.random(m)
    z = oz + L * (1.2 * rng.random(m) - 0.1)
    return np.stack([r * np.cos(ph), r * np.sin(ph), z, t], axis=1)


def field_only() -> None:
    """E of the reference's own field models on the time-dependent cases."""
    arrays, names = {}, []
    for name, kw in field_cases().items():
        pts = field_points(kw)
        arrays[f"{name}_pts"] = pts
        arrays[f"{name}_E"] = orc.harness_field(kw, pts)
        arrays[f"{name}_domain"] = json.dumps(kw)
        names.append(name)
    save("field_timed.npz", names=json.dumps(names), **arrays)


def init_state(n: int, seed: int = 123, mass_amu: float = 200.0, sigma_pos: float = 5e-4) -> dict:
    st_path = OUT / "_tmp_init.bin"
    orc.harness("init", seed=seed, n=n, sigma_pos=sigma_pos, T=300, mass=repr(mass_amu * AMU), out=st_path)
    st = orc.read_state(st_path)
    st_path.unlink()
    return st


def fticr_state(n: int) -> dict:
    """Ions on 2 mm cyclotron orbits about the trap centre (0, 0, L/2),
    m/z uniform over 500-1500 (fixed seed)."""
    rng = np.random.default_rng(7)
    m = rng.uniform(500.0, 1500.0, n) * AMU
    wc = E * 7.0 / m
    phase = rng.uniform(0, 2 * np.pi, n)
    r = 2e-3
    st = {
        "x": r * np.cos(phase) + rng.normal(0, 1e-4, n), "y": r * np.sin(phase) + rng.normal(0, 1e-4, n),
        "z": 0.025 + rng.normal(0, 1e-4, n),
        "vx": -wc * r * np.sin(phase), "vy": wc * r * np.cos(phase), "vz": rng.normal(0, 5.0, n),
        "mass": m, "charge": np.full(n, E), "ccs": np.full(n, 150e-20), "active": np.ones(n),
        "t_death": np.full(n, -1.0), "t_arrival": np.full(n, -1.0),
    }
    return st


def save(name: str, **arrays) -> None:
    np.savez_compressed(OUT / name, **arrays)
    print("wrote", name, flush=True)


def main(quick: bool, only: set[str] | None = None) -> None:
    if not orc.have_harness():
        raise SystemExit("oracle/_ref/ref_harness missing: run `make -C oracle REF=<reference tree>`")

    if only:
        if "field_timed" in only:
            field_only()
        push_only(only - {"field_timed"})
        return
    # 1. PhysicsRng streams
    streams = {}
    for seed in (123, 4219):
        p = OUT / "_u.bin"
        orc.harness("uniforms", seed=seed, n=256, out=p)
        streams[f"seed_{seed}"] = np.fromfile(p, dtype=np.float64)
        p.unlink()
    save("rng_mt64.npz", **streams)

    # 2. ion cloud
    st = init_state(64)
    save("ions_init.npz", **{k: st[k] for k in ("x", "y", "z", "vx", "vy", "vz", "mass")},
         seed=123, sigma_pos=5e-4, T=300.0, mass_amu=200.0)

    # 3. derived constants
    d = json.loads(orc.harness("derive", **IMS_DOMAIN))
    (OUT / "derived.json").write_text(json.dumps(d, indent=1) + "\n")

    # 4. collision-free pushes
    push_only(None)
    field_only()

    # 5. Boris + reference HSS, bit-level fixture for the restatement
    s0 = init_state(64)
    fin, stats, _ = orc.harness_run(s0, 2000, IMS_DOMAIN, integrator="boris", collision="hss", dt=5e-10, seed=123)
    save("hss_ref.npz", **{f"in_{k}": s0[k] for k in orc.STATE_KEYS},
         **{f"out_{k}": fin[k] for k in orc.STATE_KEYS}, steps=2000, dt=5e-10, seed=123,
         collisions=stats["collisions"], domain=json.dumps(IMS_DOMAIN))

    config0_statistics(1024 if quick else CONFIG0_IONS, 20000 if quick else 100000)


def config0_statistics(n: int, steps: int) -> None:
    """Config-0 physics run by the reference code: moments every 1000 steps,
    displacement reference after steps / 5, arrivals at z = 2 mm."""
    s0 = init_state(n)
    fin, stats, mom = orc.harness_run(s0, steps, IMS_DOMAIN, integrator="boris", collision="hss", dt=5e-10,
                                      seed=123, snap=1000, ref_step=steps // 5, zdet=2.0e-3, threads=8)
    save("ims_config0.npz", moments=mom, snap_every=1000, ref_step=steps // 5, steps=steps, dt=5e-10,
         n_ions=n, t_arrival=fin["t_arrival"], t_death=fin["t_death"], zdet=2.0e-3,
         final_vz=fin["vz"], ion_steps_per_s=stats["ion_steps_per_s"], threads=stats["threads"],
         collisions=stats["collisions"], domain=json.dumps(IMS_DOMAIN))


def push_cases() -> dict:
    return {
        "boris_ims": (IMS_DOMAIN, "boris", lambda: init_state(64), 5000, 5e-10),
        "rk4_ims": (IMS_DOMAIN, "rk4", lambda: init_state(64), 5000, 5e-10),
        "boris_fticr": (FTICR_DOMAIN, "boris", lambda: fticr_state(64), 20000, 1e-9),
        "rk4_fticr": (FTICR_DOMAIN, "rk4", lambda: fticr_state(64), 5000, 1e-9),
        "boris_quadrf": (QUAD_DOMAIN, "boris", lambda: init_state(64, mass_amu=100.0, sigma_pos=2e-4), 4000, 1e-9),
        "boris_lqit": (LQIT_DOMAIN, "boris", lambda: init_state(64, sigma_pos=2e-4), 8000, 1e-9),
        "rk4_lqit1": (LQIT1_DOMAIN, "rk4", lambda: init_state(64, sigma_pos=2e-4), 4000, 1e-9),
        "boris_tims": (TIMS_DOMAIN, "boris", lambda: init_state(64, sigma_pos=2e-4), 5000, 1e-9),
        "rk4_tims_exp": (TIMS_EXP_DOMAIN, "rk4", lambda: init_state(64, sigma_pos=2e-4), 4000, 1e-9),
        "boris_tims_wave": (TIMS_WAVE_DOMAIN, "boris", lambda: init_state(64, sigma_pos=2e-4), 5000, 1e-9),
        "boris_lqit_wave": (LQIT_WAVE_DOMAIN, "boris", lambda: init_state(64, sigma_pos=2e-4), 5000, 1e-9),
        "rk4_ims_waveref": (IMS_REF_DOMAIN, "rk4", lambda: init_state(64), 5000, 1e-9),
        "boris_quadrf_waveref": (QUAD_REF_DOMAIN, "boris", lambda: init_state(64, mass_amu=100.0, sigma_pos=2e-4),
                                 4000, 1e-9),
        "boris_ims_inline": (IMS_INLINE_DOMAIN, "boris", lambda: init_state(64), 3000, 5e-10),
        "boris_lqit_ac": (LQIT_AC_DOMAIN, "boris", lambda: init_state(64, sigma_pos=2e-4), 5000, 1e-9),
        "rk4_lqit1_ac": (LQIT1_AC_DOMAIN, "rk4", lambda: init_state(64, sigma_pos=2e-4), 4000, 1e-9),
    }


def push_only(only: set[str] | None) -> None:
    """Collision-free Boris / RK4 runs of the reference code (all, or the
    named ones)."""
    for name, (dom, integ, make_state, steps, dt) in push_cases().items():
        if only is not None and name not in only:
            continue
        s0 = make_state()
        fin, stats, _ = orc.harness_run(s0, steps, dom, integrator=integ, collision="none", dt=dt)
        save(f"push_{name}.npz", **{f"in_{k}": s0[k] for k in orc.STATE_KEYS},
             **{f"out_{k}": fin[k] for k in orc.STATE_KEYS}, steps=steps, dt=dt,
             domain=json.dumps(dom), integrator=integ)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--only", nargs="*", default=None, help="regenerate only these push fixtures (e.g. boris_lqit)")
    ap.add_argument("--config0-only", action="store_true", help="regenerate only ims_config0.npz")
    a = ap.parse_args()
    if a.config0_only:
        config0_statistics(CONFIG0_IONS, 100000)
    else:
        main(a.quick, set(a.only) if a.only else None)
