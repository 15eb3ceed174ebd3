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
        L.orc_ehss_scatter_many.argtypes = [C.c_int64, DP, DP, C.c_double, C.c_double, C.c_uint64, DP]
        L.orc_set_ipm_table.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_double, C.c_double]
        L.orc_ipm_cos_chi_trajectory.argtypes = [C.c_double] * 7
        L.orc_ipm_cos_chi_trajectory.restype = C.c_double
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


def mt64_uniforms(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    lib().orc_mt64_uniforms(seed, n, _dp(out))
    return out


def philox(ctr: np.ndarray, seed: int) -> np.ndarray:
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    key = np.array([seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF], dtype=np.uint32)
    out = np.zeros_like(ctr)
    P = C.POINTER(C.c_uint32)
    lib().orc_philox_many(ctr.shape[0], ctr.ctypes.data_as(P), key.ctypes.data_as(P), out.ctypes.data_as(P))
    return out


def run(domain: dict, state: dict, n_steps: int, *, integrator: int = 0, collision: int = 0, seed: int = 123,
        first_id: int = 0, step0: int = 0, t0: float = 0.0, snap_every: int = 0, ref_step: int = 0,
        clock: tuple | None = None, threads: int = 1, subcycles: int = 1) -> dict:
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
    skip clock)."""
    d = domain_struct(domain)
    lib().orc_set_subcycles(int(subcycles))
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
