"""Transport observables from snapshot moments (definitions shared by the
device runs, the CPU oracle runs and the reference-code runs).

* mean drift velocity v_d: least-squares slope of <dz>(t) over the fit window
  (same fit-window idea as validation/scripts/physics/measure_K0_directly.py:114-141)
* K0 = (v_d / E) * (N / N0), N0 = 101325 / (kB 273.15)  (measure_K0_directly.py:171-174)
* D_L = 1/2 d Var(dz)/dt, D_T = 1/4 d[Var(dx) + Var(dy)]/dt, with dx the
  displacement from the reference positions (start of the fit window)
* arrival times: first crossing of the detector plane, compared with a
  two-sample Kolmogorov-Smirnov test

Moments layout: include/icarion_b200.h (ICB_N_MOMENTS).
"""
from __future__ import annotations

import math

import numpy as np

from . import config as cfgmod


def _slope(t: np.ndarray, y: np.ndarray) -> float:
    tm = t.mean()
    return float(np.sum((t - tm) * (y - y.mean())) / np.sum((t - tm) ** 2))


def fit_transport(times: np.ndarray, mom: np.ndarray, t_ref: float) -> dict:
    """times [S], mom [S, 20] of one ensemble; snapshots with t >= t_ref are
    fitted (the displacement reference was taken at t_ref)."""
    sel = times >= t_ref - 1e-18
    t = times[sel] - t_ref
    m = mom[sel]
    n = m[:, 0]
    if np.any(n <= 1):
        raise ValueError("not enough active ions in the fit window")
    mdx, mdy, mdz = m[:, 14] / n, m[:, 15] / n, m[:, 16] / n
    vxx = m[:, 17] / n - mdx ** 2
    vyy = m[:, 18] / n - mdy ** 2
    vzz = m[:, 19] / n - mdz ** 2
    vd = _slope(t, mdz)
    dl = 0.5 * _slope(t, vzz)
    dt_ = 0.25 * _slope(t, vxx + vyy)
    N = float(n[-1])
    T = float(t[-1] - t[0]) if len(t) > 1 else float(t[-1])
    # statistical standard errors of the window estimators (independent ions):
    # Var(<dz>) = 2 D_L T / N  -> se(v_d) ~ sqrt(2 D_L / (N T));  se(D)/D ~ sqrt(2/N)
    se_vd = math.sqrt(max(2.0 * dl, 0.0) / (N * T)) if T > 0 else float("nan")
    return {
        "v_drift": vd, "D_L": dl, "D_T": dt_, "n_ions": N,
        "se_v_drift": se_vd, "se_D_L": abs(dl) * math.sqrt(2.0 / N), "se_D_T": abs(dt_) * math.sqrt(1.0 / N),
        "mean_speed2": float(m[-1, 10] / n[-1]),
    }


def k0_from_drift(v_drift: float, e_field: float, gas_density: float) -> float:
    """Reduced mobility in cm^2/(V s)."""
    return (v_drift / e_field) * (gas_density / cfgmod.n0_loschmidt()) * 1e4


def ks_2samp(a: np.ndarray, b: np.ndarray) -> tuple[float, float]:
    """Two-sample Kolmogorov-Smirnov statistic and p-value."""
    from scipy import stats
    r = stats.ks_2samp(np.asarray(a), np.asarray(b))
    return float(r.statistic), float(r.pvalue)


def rel_err(a: float, b: float) -> float:
    return abs(a - b) / abs(b)
