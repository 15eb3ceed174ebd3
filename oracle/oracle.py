"""ORACLE — test infrastructure only (the checker, never the product).

Python access to
  * ``liboracle.so`` — the C restatement of the reference's batch step
    (``icb_oracle.c``), and
  * ``_ref/ref_harness`` — the reference's own sources compiled by
    ``oracle/Makefile`` (present where the reference tree was available at
    build time; the binary travels with the repository snapshot).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
HARNESS = HERE / "_ref" / "ref_harness"
N_MOMENTS = 20

D3 = C.c_double * 3


class Domain(C.Structure):
    """orc_domain (same layout as icb_ensemble_params)."""
    _fields_ = [
        ("instrument", C.c_int32), ("magnetic_enabled", C.c_int32),
        ("origin_m", D3), ("length_m", C.c_double), ("radius_m", C.c_double),
        ("axial_V", C.c_double), ("radial_V", C.c_double), ("dc_quad_V", C.c_double),
        ("rf_voltage_V", C.c_double), ("rf_frequency_Hz", C.c_double), ("B_T", D3),
        ("temperature_K", C.c_double), ("gas_density_m3", C.c_double), ("gas_mass_kg", C.c_double),
        ("gas_velocity_m_s", D3), ("gas_polarizability_m3", C.c_double), ("sigma_m2", C.c_double),
        ("ipm_bmax_m", C.c_double), ("dt_s", C.c_double), ("detector_z_m", C.c_double),
        ("n_gas", C.c_int32), ("flow_model", C.c_int32), ("gas_mix_density_m3", C.c_double * 8),
        ("gas_mix_mass_kg", C.c_double * 8), ("gas_mix_sigma_m2", C.c_double * 8),
        ("axial_flow_velocity_m_s", C.c_double), ("axial_flow_max_velocity_m_s", C.c_double),
        ("ac_amplitude_V", C.c_double * 2), ("ac_frequency_Hz", C.c_double * 2), ("ac_phase_rad", C.c_double * 2),
        ("ac_ramp", C.c_double * 2), ("ac_dipolar", C.c_int32), ("reserved2_", C.c_int32),
    ]


class OWave(C.Structure):
    """orc_wave (same layout as icb_waveform)."""
    _fields_ = [("type", C.c_int32), ("clamp", C.c_int32), ("interp", C.c_int32), ("n_points", C.c_int32),
                ("p", C.c_double * 8), ("times_s", C.c_double * 64), ("values", C.c_double * 64)]


class OTims(C.Structure):
    """orc_tims (same layout as icb_tims_field)."""
    _fields_ = [("ramp_mode", C.c_int32), ("n_nodes", C.c_int32), ("has_final_profile", C.c_int32),
                ("reserved_", C.c_int32), ("ei", C.c_double), ("ef", C.c_double), ("t0", C.c_double),
                ("t1", C.c_double), ("tau", C.c_double), ("z", C.c_double * 64), ("pi", C.c_double * 64),
                ("pf", C.c_double * 64)]


WAVE_KEYS = ("wave_axial", "wave_quad", "wave_rfv", "wave_rff", "wave_ramp",
             "wave_acxA", "wave_acxf", "wave_acxr", "wave_acyA", "wave_acyf", "wave_acyr")


def parse_wave(spec: str) -> dict:
    """Harness waveform spec "type|clamp|interp|p0,..|t0,..|v0,.." -> fields."""
    f = (str(spec).split("|") + [""] * 6)[:6]
    num = lambda x: [float(v) for v in x.split(",") if v != ""]
    p = (num(f[3]) + [0.0] * 8)[:8]
    return {"type": int(f[0]), "clamp": int(f[1] or 0), "interp": int(f[2] or 0), "p": p,
            "times": num(f[4]), "values": num(f[5])}


def wave_struct(spec: str, cls=OWave):
    d = parse_wave(spec)
    w = cls()
    w.type, w.clamp, w.interp = d["type"], d["clamp"], d["interp"]
    w.n_points = len(d["times"]) if d["type"] == 7 else 0
    w.p[:] = d["p"]
    w.times_s[:len(d["times"])] = d["times"]
    w.values[:len(d["values"])] = d["values"]
    return w


def tims_struct(kw: dict, cls=OTims, names=("ei", "ef", "t0", "t1", "tau", "z", "pi", "pf")):
    """Harness TIMS keys -> orc_tims (or the ABI struct with its field names)."""
    if not kw.get("tims"):
        return None
    num = lambda x: [float(v) for v in str(x).split(",") if v != ""]
    t = cls()
    t.ramp_mode = int(kw.get("tims_mode", 0))
    z, pi, pf = num(kw.get("tims_z", "")), num(kw.get("tims_pi", "")), num(kw.get("tims_pf", ""))
    t.n_nodes = len(z)
    t.has_final_profile = int(len(pf) == len(z) and len(z) > 0)
    ei, ef, t0, t1, tau, zf, pif, pff = names
    setattr(t, ei, float(kw.get("tims_ei", 0.0)))
    setattr(t, ef, float(kw.get("tims_ef", 0.0)))
    setattr(t, t0, float(kw.get("tims_t0", 0.0)))
    setattr(t, t1, float(kw.get("tims_t1", 0.0)))
    setattr(t, tau, float(kw.get("tims_tau", 1e-3)))
    getattr(t, zf)[:len(z)] = z
    getattr(t, pif)[:len(pi)] = pi
    getattr(t, pff)[:len(pf)] = pf
    return t


def wave_value(spec: str, t: float) -> float:
    """The restated waveform evaluation at one time."""
    w = wave_struct(spec)
    return lib().orc_wave_value(C.byref(w), float(t))


def set_time_field(kw: dict | None) -> None:
    """Waveforms and TIMS field of the harness domain keys (None clears)."""
    kw = kw or {}
    waves = (OWave * len(WAVE_KEYS))()
    on = (C.c_int32 * len(WAVE_KEYS))()
    for c, key in enumerate(WAVE_KEYS):
        if key in kw:
            waves[c] = wave_struct(kw[key])
            on[c] = 1
    t = tims_struct(kw)
    lib().orc_set_time_field(C.byref(t) if t is not None else None, waves, on)


def field(domain: dict, pts: np.ndarray, time_field: dict | None = None) -> np.ndarray:
    """E of the restated field model at rows (x, y, z, t)."""
    d = domain_struct(domain)
    set_time_field(time_field)
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 4)
    out = np.zeros((pts.shape[0], 3))
    for i in range(pts.shape[0]):
        p = np.ascontiguousarray(pts[i, :3])
        e = np.zeros(3)
        lib().orc_field(C.byref(d), _dp(p), float(pts[i, 3]), _dp(e))
        out[i] = e
    return out


def domain_struct(p: dict) -> Domain:
    d = Domain()
    for k, _ in Domain._fields_:
        v = p[k]
        if isinstance(v, (list, tuple)):
            getattr(d, k)[:] = [float(x) for x in v]
        else:
            setattr(d, k, v)
    return d


_lib = None


def build() -> None:
    """make -C oracle (restatement always; reference harness if the
    reference tree is present)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, capture_output=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        DP = C.POINTER(C.c_double)
        U8P = C.POINTER(C.c_uint8)
        U32P = C.POINTER(C.c_uint32)
        U64P = C.POINTER(C.c_uint64)
        L.orc_mt64_uniforms.argtypes = [C.c_uint64, C.c_int64, DP]
        L.orc_philox4x32_10.argtypes = [U32P, U32P, U32P]
        L.orc_philox_many.argtypes = [C.c_int64, U32P, U32P, U32P]
        L.orc_philox2x32_10.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, U32P]
        L.orc_step_test_word.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32]
        L.orc_step_test_word.restype = C.c_uint32
        L.orc_unit_uniforms.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, DP]
        L.orc_field.argtypes = [C.POINTER(Domain), DP, C.c_double, DP]
        L.orc_clock_init.argtypes = [C.c_uint64, C.c_int64, C.c_uint64, DP, DP, U32P, U32P, C.c_int]
        L.orc_field_bound.argtypes = [C.POINTER(Domain)]
        L.orc_field_bound.restype = C.c_double
        L.orc_thermal_width.argtypes = [C.c_double, C.c_double]
        L.orc_thermal_width.restype = C.c_double
        L.orc_run.argtypes = [C.POINTER(Domain), C.c_int, C.c_int, C.c_uint64, C.c_int64,
                              DP, DP, DP, DP, DP, DP, DP, DP, U8P, DP, DP, DP, DP, U32P, U32P,
                              C.c_uint64, C.c_uint64, C.c_double, C.c_int64, C.c_int64, C.c_int64,
                              DP, U64P, C.c_int]
        L.orc_run.restype = C.c_int
        L.orc_set_ehss.argtypes = [DP, C.c_int, C.c_double]
        L.orc_set_subcycles.argtypes = [C.c_int]
        L.orc_set_time_field.argtypes = [C.POINTER(OTims), C.POINTER(OWave), C.POINTER(C.c_int32)]
        L.orc_wave_value.argtypes = [C.POINTER(OWave), C.c_double]
        L.orc_wave_value.restype = C.c_double
        L.orc_ehss_scatter_many.argtypes = [C.c_int64, DP, DP, C.c_double, C.c_double, C.c_uint64, DP]
        L.orc_set_ipm_table.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_ipm_cos_chi_trajectory.argtypes = [C.c_double] * 7
        L.orc_ipm_cos_chi_trajectory.restype = C.c_double
        L.orc_ipm_chi_quad.argtypes = [C.c_double] * 6
        L.orc_ipm_chi_quad.restype = C.c_double
        L.orc_ipm_cos_chi_many.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double, DP, DP, DP]
        L.orc_ipm_sample_cells.argtypes = [C.c_int64, DP] + [C.c_double] * 6 + [C.c_int64, C.c_uint64, C.c_int, DP]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _u32(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_uint32))


_ipm_table_ref = None


def set_ipm_table(tab: np.ndarray, n_E: int, n_b: int, ln_E_min: float, inv_dlnE: float) -> None:
    """Interaction-potential table for collision model 4 (kept alive here)."""
    global _ipm_table_ref
    _ipm_table_ref = np.ascontiguousarray(tab, dtype=np.float32)
    lib().orc_set_ipm_table(_ipm_table_ref.ctypes.data_as(C.POINTER(C.c_float)), n_E, n_b, ln_E_min, inv_dlnE)


_ehss_ref = None


def set_ehss(atoms: np.ndarray, gas_radius: float) -> None:
    """EHSS geometry (n x 4: x, y, z, r) for collision model 7 (kept alive here)."""
    global _ehss_ref
    _ehss_ref = np.ascontiguousarray(atoms, dtype=np.float64).reshape(-1, 4)
    lib().orc_set_ehss(_dp(_ehss_ref.ravel()), _ehss_ref.shape[0], gas_radius)


def ehss_scatter_many(v_ion: np.ndarray, v_n: np.ndarray, mi: float, mn: float, seed: int) -> np.ndarray:
    """The restated EHSS scattering of n ions (geometry from set_ehss)."""
    vi = np.ascontiguousarray(v_ion, dtype=np.float64).reshape(-1, 3)
    vn = np.ascontiguousarray(v_n, dtype=np.float64).reshape(-1, 3)
    out = np.zeros_like(vi)
    lib().orc_ehss_scatter_many(vi.shape[0], _dp(vi.ravel()), _dp(vn.ravel()), mi, mn, seed, _dp(out.ravel()))
    return out


def harness_ehss(atoms: np.ndarray, gas_radius: float, v_ion: np.ndarray, v_n: np.ndarray, mi: float, mn: float,
                 seed: int = 1) -> np.ndarray:
    """The reference's own CollisionKernels::ehss_collision on the same inputs."""
    at = np.ascontiguousarray(atoms, dtype=np.float64).reshape(-1, 4)
    vi = np.ascontiguousarray(v_ion, dtype=np.float64).reshape(-1, 3)
    vn = np.ascontiguousarray(v_n, dtype=np.float64).reshape(-1, 3)
    with tempfile.TemporaryDirectory() as td:
        ip, op = Path(td) / "in.bin", Path(td) / "out.bin"
        with open(ip, "wb") as f:
            f.write(np.int64(at.shape[0]).tobytes())
            f.write(at.tobytes())
            f.write(np.int64(vi.shape[0]).tobytes())
            f.write(vi.tobytes())
            f.write(vn.tobytes())
        harness("ehss", **{"in": ip, "out": op, "mi": repr(mi), "mn": repr(mn), "rgas": repr(gas_radius),
                           "seed": seed})
        return np.fromfile(op, dtype=np.float64).reshape(-1, 3)


def ipm_cos_chi_trajectory(c12: float, c6: float, c4: float, m_red: float, E: float, b: float,
                           max_step_m: float = 0.05e-10) -> float:
    """cos(chi) from the restated reference trajectory integrator."""
    return lib().orc_ipm_cos_chi_trajectory(c12, c6, c4, m_red, E, b, max_step_m)


def ipm_cos_chi_quad(c12: float, c6: float, c4: float, sigma: float, E: np.ndarray, b: np.ndarray) -> np.ndarray:
    """cos(chi) of the restated deflection quadrature at (E, b) pairs."""
    E = np.ascontiguousarray(E, dtype=np.float64).ravel()
    b = np.ascontiguousarray(np.broadcast_to(b, E.shape), dtype=np.float64)
    out = np.zeros_like(E)
    lib().orc_ipm_cos_chi_many(E.size, c12, c6, c4, sigma, _dp(E), _dp(b), _dp(out))
    return out


def ipm_table(c12: float, c6: float, c4: float, sigma: float, n_E: int, n_b: int, E_min: float, E_max: float,
              b_max: float) -> np.ndarray:
    """The handle's cos(chi) table on the CPU: float32 [n_E, n_b] at
    E_k = E_min (E_max / E_min)^(k / (n_E - 1)), b_j = b_max j / (n_b - 1)."""
    import math
    dlnE = (math.log(E_max) - math.log(E_min)) / (n_E - 1)
    E = np.repeat(np.exp(math.log(E_min) + np.arange(n_E) * dlnE), n_b)
    b = np.tile(np.arange(n_b) * (b_max / (n_b - 1)), n_E)
    return ipm_cos_chi_quad(c12, c6, c4, sigma, E, b).astype(np.float32).reshape(n_E, n_b)


def ipm_sample_cells(c12: float, c6: float, c4: float, sigma: float, mu: float, g: np.ndarray, b_max: float,
                     n_trials: int, seed: int, stratified: bool = True) -> np.ndarray:
    """Momentum-transfer samples of sample-set cells at relative speeds g
    ((len(g), n_trials, 3)): the reference tool's per-cell rule with the
    restated quadrature; stratified = True takes the impact points from
    equal-area annuli (same law, no Monte Carlo noise in the cell means)."""
    g = np.ascontiguousarray(g, dtype=np.float64)
    dp = np.zeros(3 * n_trials * g.size)
    lib().orc_ipm_sample_cells(g.size, _dp(g), c12, c6, c4, sigma, mu, b_max, n_trials, seed, int(stratified),
                               _dp(dp))
    return dp.reshape(g.size, n_trials, 3)


def write_ipm_sample_set(path: Path, c12: float, c6: float, c4: float, sigma: float, mu: float, g_min: float,
                         g_max: float, n_bins: int, b_max: float, n_trials: int, seed: int, stratified: bool = True,
                         gas: str = "N2") -> dict:
    """The reference's offline sample set (InteractionPotentialOfflineSampleSet
    .h:16-98: one orientation, n_bins log-spaced relative speeds, a fixed
    event disk of radius b_max, full momentum-transfer CDFs with equal
    weights, interaction_potential_precompute.cpp:2692-2880) in the flat file
    layout read by oracle/ref_ipm_loader.cpp.  Returns the per-bin summary."""
    logv = np.linspace(np.log(g_min), np.log(g_max), n_bins)
    g = np.exp(logv)
    dps = ipm_sample_cells(c12, c6, c4, sigma, mu, g, b_max, n_trials, seed, stratified)
    one_minus_cos = -dps[:, :, 2] / (mu * g[:, None])
    smt = np.pi * b_max ** 2 * one_minus_cos.mean(axis=1)
    perp = np.hypot(dps[:, :, 0], dps[:, :, 1])
    stats = np.stack([dps[:, :, 2].mean(axis=1), perp.mean(axis=1), dps[:, :, 2].var(axis=1), perp.var(axis=1)],
                     axis=1)
    cells = n_bins
    sev = np.full(cells, np.pi * b_max ** 2)
    offsets = np.arange(cells, dtype=np.int64) * n_trials
    counts = np.full(cells, n_trials, dtype=np.int64)
    cdf = np.tile((np.arange(n_trials) + 1.0) / n_trials, cells)
    gb = gas.encode()
    with open(path, "wb") as f:
        f.write(b"ICBIPMS1")
        f.write(np.array([1, n_bins, cells * n_trials, len(gb)], dtype=np.int64).tobytes())
        f.write(gb)
        for arr in (logv, smt, sev, np.full(cells, b_max)):
            f.write(np.ascontiguousarray(arr, dtype=np.float64).tobytes())
        f.write(offsets.tobytes())
        f.write(counts.tobytes())
        f.write(cdf.astype(np.float64).tobytes())
        f.write(np.ascontiguousarray(dps, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(stats, dtype=np.float64).tobytes())
    return {"logv_bins": logv, "sigma_mt_m2": smt, "sigma_event_m2": sev}


def mt64_uniforms(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    lib().orc_mt64_uniforms(seed, n, _dp(out))
    return out


def philox2x32(c0: int, c1: int, key: int) -> tuple[int, int]:
    """Philox2x32-10 of the counter (c0, c1) under `key` (both words)."""
    out = (C.c_uint32 * 2)()
    lib().orc_philox2x32_10(c0, c1, key, out)
    return int(out[0]), int(out[1])


def step_test_word(seed: int, step: int, ion_id: int) -> int:
    """The per-step kernel's collision-test word of (step, ion id)."""
    return int(lib().orc_step_test_word(seed, step, ion_id))


def philox(ctr: np.ndarray, seed: int) -> np.ndarray:
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    key = np.array([seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF], dtype=np.uint32)
    out = np.zeros_like(ctr)
    P = C.POINTER(C.c_uint32)
    lib().orc_philox_many(ctr.shape[0], ctr.ctypes.data_as(P), key.ctypes.data_as(P), out.ctypes.data_as(P))
    return out


def run(domain: dict, state: dict, n_steps: int, *, integrator: int = 0, collision: int = 0, seed: int = 123,
        first_id: int = 0, step0: int = 0, t0: float = 0.0, snap_every: int = 0, ref_step: int = 0,
        clock: tuple | None = None, threads: int = 1, subcycles: int = 1,
        time_field: dict | None = None) -> dict:
    """Run the restatement.  ``state`` holds float64 arrays x..vz, mass, charge,
    uint8 active and optional t_death / t_arrival; it is updated in place.
    collision: 0 none, 1 reference HSS (mt19937_64 per ion), 2 null-collision
    HSS with Philox (``clock`` = (S, U, next, start) arrays from a previous
    call, or None to initialise; Boris uses the skip clock, RK4 the per-step
    clock), 3 Langevin capture with Philox (Boris, skip clock), 4
    interaction-potential table collisions (Boris, skip clock; table from
    set_ipm_table), 5 HSS gas mixture (Boris, skip clock), 6 the reference's
    per-step HSS form with Philox words (no clock; ``subcycles`` collision
    sub-steps of dt/m per step), 7 EHSS on the geometry of set_ehss (Boris,
    skip clock), 8 null-collision HSS with the per-step kernel's stateless
    test (Boris; no clock state).  ``time_field`` holds the harness's waveform / TIMS keys
    (wave_*, tims*) of the domain; the default clears them."""
    d = domain_struct(domain)
    lib().orc_set_subcycles(int(subcycles))
    set_time_field(time_field)
    n = state["x"].shape[0]
    for k in ("t_death", "t_arrival"):
        if state.get(k) is None:
            state[k] = np.full(n, -1.0)
    S = U = nxt = start = None
    if collision in (2, 3, 4, 5, 7):
        if clock is None:
            S, U = np.zeros(n), np.zeros(n)
            nxt, start = np.zeros(n, dtype=np.uint32), np.zeros(n, dtype=np.uint32)
            lib().orc_clock_init(seed, n, first_id, _dp(S), _dp(U), _u32(nxt), _u32(start), 1 if integrator == 0 else 0)
        else:
            S, U, nxt, start = clock
    n_snap = n_steps // snap_every if snap_every > 0 else 0
    mom = np.zeros((max(n_snap, 1), N_MOMENTS))
    cnt = np.zeros(3, dtype=np.uint64)
    rc = lib().orc_run(C.byref(d), integrator, collision, seed, n,
                       _dp(state["x"]), _dp(state["y"]), _dp(state["z"]),
                       _dp(state["vx"]), _dp(state["vy"]), _dp(state["vz"]),
                       _dp(state["mass"]), _dp(state["charge"]),
                       state["active"].ctypes.data_as(C.POINTER(C.c_uint8)),
                       _dp(state["t_death"]), _dp(state["t_arrival"]), _dp(S), _dp(U), _u32(nxt), _u32(start),
                       first_id, step0, t0, n_steps, snap_every, ref_step,
                       _dp(mom) if n_snap else None, cnt.ctypes.data_as(C.POINTER(C.c_uint64)), threads)
    if rc != 0:
        raise RuntimeError(f"orc_run failed ({rc})")
    return {"moments": mom[:n_snap], "candidates": int(cnt[0]), "collisions": int(cnt[1]),
            "rate_overflows": int(cnt[2]), "clock": (S, U, nxt, start)}


# ---------------------------------------------------------------------------
# reference harness (the reference's own code)
# ---------------------------------------------------------------------------
STATE_KEYS = ("x", "y", "z", "vx", "vy", "vz", "mass", "charge", "ccs", "active", "t_death", "t_arrival")


def have_harness() -> bool:
    return HARNESS.exists()


def write_state(path: Path, st: dict) -> None:
    n = st["x"].shape[0]
    with open(path, "wb") as f:
        f.write(np.int64(n).tobytes())
        for k in STATE_KEYS:
            v = st.get(k)
            if v is None:
                v = np.full(n, -1.0) if k in ("t_death", "t_arrival") else np.zeros(n)
            f.write(np.ascontiguousarray(v, dtype=np.float64).tobytes())


def read_state(path: Path) -> dict:
    raw = Path(path).read_bytes()
    n = int(np.frombuffer(raw[:8], dtype=np.int64)[0])
    arr = np.frombuffer(raw[8:], dtype=np.float64).reshape(len(STATE_KEYS), n)
    st = {k: arr[i].copy() for i, k in enumerate(STATE_KEYS)}
    st["active"] = st["active"].astype(np.uint8)
    return st


def harness(mode: str, **kw) -> str:
    args = [str(HARNESS), mode] + [f"{k}={v}" for k, v in kw.items()]
    env = dict(os.environ)
    env.setdefault("OMP_PLACES", "cores")
    env.setdefault("OMP_PROC_BIND", "close")
    r = subprocess.run(args, capture_output=True, text=True, env=env)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness {mode} failed: {r.stderr}")
    return r.stdout


def harness_field(domain_kw: dict, pts: np.ndarray) -> np.ndarray:
    """E of the reference's own field model (the one PhysicsSetup builds for
    the domain) at rows (x, y, z, t)."""
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 4)
    with tempfile.TemporaryDirectory() as td:
        ip, op = Path(td) / "pts.bin", Path(td) / "E.bin"
        ip.write_bytes(pts.tobytes())
        harness("field", **{"in": ip, "out": op}, **domain_kw)
        return np.fromfile(op, dtype=np.float64).reshape(-1, 3)


def harness_run(state: dict, n_steps: int, domain_kw: dict, **kw) -> tuple[dict, dict, np.ndarray | None]:
    """Run the reference code on ``state``; returns (final state, json stats, moments)."""
    with tempfile.TemporaryDirectory() as td:
        ip, op, mp = Path(td) / "in.bin", Path(td) / "out.bin", Path(td) / "mom.bin"
        write_state(ip, state)
        out = harness("run", **{"in": ip, "out": op, "mom": mp, "steps": n_steps}, **domain_kw, **kw)
        stats = json.loads(out.strip().splitlines()[-1])
        st = read_state(op)
        mom = np.fromfile(mp, dtype=np.float64).reshape(-1, N_MOMENTS) if mp.exists() else None
    return st, stats, mom
