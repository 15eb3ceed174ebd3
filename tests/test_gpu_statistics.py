"""Stochastic parity of the fused kernel.

1. Config-0 physics (100,000 steps, Boris + HSS, 20 Td) on 65,536 ions:
   FP64 and mixed device runs against the reference's own CPU code (golden
   ims_config0.npz, same initial cloud): drift velocity, K0, D_L, D_T
   within 4 combined standard errors (at this size ~0.04 % on K0, ~0.6 %
   on D_L and D_T per run); collision fraction within 0.3 %; arrival-time
   distributions at z = 2 mm with a two-sample KS p-value > 0.01.
2. Config 1 physics at 1,048,576 ions: mixed and hi/lo mixed against the
   FP64 device form (the FP64 oracle run): K0 within 0.3 %, D_L and D_T
   within 1 %.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import config0_ensemble, config0_ions
from icarion_b200 import _capi as capi
from icarion_b200 import observables as ob
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu

DT = 5e-10
E_Z = 4828.6470106932802
N_GAS = 2.4143235053466402e23


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def device_run(n: int, steps: int, precision: int, snap: int = 1000, ref_step: int = 20000):
    e = config0_ensemble(detector_z_m=2.0e-3, dt=DT)
    st0 = config0_ions(n)
    with Simulation([e], precision=precision, integrator=capi.INTEGRATOR_BORIS, collision=capi.COLLISION_HSS,
                    rng_seed=123) as sim:
        sim.upload(st0)
        steps_idx, mom, tot = sim.run(steps, snap, ref_step=ref_step)
        fin = sim.download()
    t = steps_idx * DT
    fit = ob.fit_transport(t, mom[:, 0, :], t_ref=ref_step * DT)
    fit["K0"] = ob.k0_from_drift(fit["v_drift"], E_Z, N_GAS)
    fit["se_K0"] = fit["K0"] * fit["se_v_drift"] / fit["v_drift"]
    return fit, fin, tot


def reference_fit(golden):
    z = golden("ims_config0.npz")
    mom = z["moments"]
    t = np.arange(1, mom.shape[0] + 1) * int(z["snap_every"]) * float(z["dt"])
    fit = ob.fit_transport(t, mom, t_ref=int(z["ref_step"]) * float(z["dt"]))
    fit["K0"] = ob.k0_from_drift(fit["v_drift"], E_Z, N_GAS)
    fit["se_K0"] = fit["K0"] * fit["se_v_drift"] / fit["v_drift"]
    return fit, z


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_config0_observables_match_reference_cpu(golden, precision):
    ref, z = reference_fit(golden)
    n = int(z["n_ions"])
    assert n >= 4096 and int(z["steps"]) == 100000
    fit, fin, tot = device_run(n, 100000, precision)
    for key in ("v_drift", "K0", "D_L", "D_T"):
        se = np.hypot(ref["se_" + key], fit["se_" + key])
        assert abs(fit[key] - ref[key]) <= 4.0 * se, (key, fit[key], ref[key], se)
    # collision fraction of ion-steps (reference: collisions / (N * steps))
    f_ref = float(z["collisions"]) / (n * 100000)
    f_dev = tot["collisions"] / (n * 100000)
    assert abs(f_dev - f_ref) / f_ref < 0.003, (f_dev, f_ref)
    a, b = fin.t_arrival[fin.t_arrival >= 0], z["t_arrival"][z["t_arrival"] >= 0]
    assert abs(len(a) - len(b)) <= 0.01 * n
    _, p = ob.ks_2samp(a, b)
    assert p > 0.01, p


def test_mixed_precision_accuracy_at_1M_ions():
    """Also prints the measured differences (one JSON line per float form):
    relative difference and its combined standard error for v_drift, K0,
    D_L, D_T, and the two-sample KS p-value of the arrival times."""
    import json
    n = 1_048_576
    fp64, fin64, _ = device_run(n, 100000, capi.PREC_FP64)
    a64 = fin64.t_arrival[fin64.t_arrival >= 0]
    for prec in (capi.PREC_MIXED, capi.PREC_MIXED_HILO):
        mix, fin, _ = device_run(n, 100000, prec)
        row = {"form": {capi.PREC_MIXED: "mixed", capi.PREC_MIXED_HILO: "hilo"}[prec], "ions": n, "steps": 100000}
        for key in ("v_drift", "K0", "D_L", "D_T"):
            row[key] = {"rel_diff": (mix[key] - fp64[key]) / fp64[key],
                        "rel_se": float(np.hypot(mix["se_" + key], fp64["se_" + key])) / abs(fp64[key])}
        a = fin.t_arrival[fin.t_arrival >= 0]
        row["arrivals"] = {"fp64": int(len(a64)), "form": int(len(a)), "ks_p": float(ob.ks_2samp(a, a64)[1])}
        print("precision accuracy:", json.dumps(row))
        assert ob.rel_err(mix["K0"], fp64["K0"]) <= 3e-3, (prec, mix["K0"], fp64["K0"])
        assert ob.rel_err(mix["D_L"], fp64["D_L"]) <= 1e-2, (prec, mix["D_L"], fp64["D_L"])
        assert ob.rel_err(mix["D_T"], fp64["D_T"]) <= 1e-2, (prec, mix["D_T"], fp64["D_T"])
