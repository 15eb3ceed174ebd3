"""The batched E/N sweep at its own settings (50,000 steps, dt = 0.1 /
nu_max per ensemble).

1. One ensemble of each species (30, 31, 32: 12.9 / 13.7 / 14.6 Td with
   (100 Da, 100 A^2), (500 Da, 250 A^2), (2000 Da, 600 A^2)) against the
   reference's own Boris + HSS code (fixture sweep_ref.npz, 4,096 ions):
   v_drift, K0, D_L, D_T within 4 combined standard errors, collision
   fraction within 1 %, FP64 and mixed.
2. The whole sweep (64 ensembles, 2-100 Td, the three species round-robin)
   with 655,360 ions per ensemble: mixed against FP64 per ensemble.  The
   runs are statistically independent (float rounding decorrelates the
   ions' collision sequences), so each difference carries the standard
   error of both runs, stated by the fit: for D_L and D_T ~0.25 %
   (sqrt(2/N) each), for K0 from 0.01 % at 100 Td to ~0.8 % at 2 Td (at
   50,000 steps of dt = 0.1 / nu_max the low-field ensembles drift only a
   few um against ~20 um of diffusion).  Gates: K0 within max(0.3 %, 4
   standard errors of the difference), D_L and D_T within max(1 %, 4
   standard errors), and no bias over the sweep: the mean squared
   normalised difference of each observable below 4 (1 when the stated
   errors are exact; a shift of two standard errors in every ensemble
   gives 5).
"""
from __future__ import annotations

import json

import numpy as np
import pytest

from helpers import assert_transport_close, domain_json, ion_cloud
from icarion_b200 import _capi as capi
from icarion_b200 import config as cfg
from icarion_b200 import observables as ob
from icarion_b200 import sweep
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def fits_of(ensembles, steps_idx, mom, ref_step):
    out = []
    for e, E in enumerate(ensembles):
        t = steps_idx * E["dt_s"]
        f = ob.fit_transport(t, mom[:, e, :], t_ref=ref_step * E["dt_s"])
        f["K0"] = ob.k0_from_drift(f["v_drift"], E["axial_V"] / E["length_m"], E["gas_density_m3"])
        f["se_K0"] = f["K0"] * f["se_v_drift"] / f["v_drift"]
        out.append(f)
    return out


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_one_ensemble_per_species_matches_reference_code(golden, precision):
    z = golden("sweep_ref.npz")
    n, steps, snap, ref = int(z["n_ions"]), int(z["steps"]), int(z["snap_every"]), int(z["ref_step"])
    for e in z["ensembles"]:
        p = f"e{int(e)}_"
        E = cfg.ensemble_params(domain_json(json.loads(str(z[p + "domain"]))), float(z[p + "ccs_a2"]) * 1e-20,
                                float(z[p + "dt"]), detector_z_m=2.0e-3)
        st0 = ion_cloud(n, float(z[p + "mass_amu"]), int(z["seed"]))
        with Simulation([E], precision=precision, collision=capi.COLLISION_HSS, rng_seed=int(z["seed"])) as sim:
            sim.upload(st0)
            steps_idx, mom, tot = sim.run(steps, snap, ref_step=ref)
        ref_mom = z[p + "moments"]
        got = fits_of([E], steps_idx, mom, ref)[0]
        want = fits_of([E], steps_idx, ref_mom[:, None, :], ref)[0]
        assert_transport_close(got, want)
        f_ref = float(z[p + "collisions"]) / (n * steps)
        assert abs(tot["collisions"] / (n * steps) / f_ref - 1.0) < 0.01, (int(e), tot["collisions"], f_ref)


def test_whole_sweep_mixed_matches_fp64_per_ensemble():
    sw = sweep.en_sweep(n_ensembles=64, counts=np.full(64, 655_360))
    steps, snap, ref = 50_000, 1_000, 10_000
    fits = {}
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        with Simulation(sw.ensembles, precision=prec, collision=capi.COLLISION_HSS, rng_seed=123) as sim:
            sim.upload(sw.ions, ens_offsets=sw.offsets)
            steps_idx, mom, _ = sim.run(steps, snap, ref_step=ref)
        fits[prec] = fits_of(sw.ensembles, steps_idx, mom, ref)
    worst = {"K0": 0.0, "D_L": 0.0, "D_T": 0.0}
    chi2 = {"K0": 0.0, "D_L": 0.0, "D_T": 0.0}
    for e in range(64):
        a, b = fits[capi.PREC_MIXED][e], fits[capi.PREC_FP64][e]
        for key, tol in (("K0", 3e-3), ("D_L", 1e-2), ("D_T", 1e-2)):
            r = ob.rel_err(a[key], b[key])
            se = float(np.hypot(a["se_" + key], b["se_" + key])) / abs(b[key])
            worst[key] = max(worst[key], r)
            chi2[key] += (r / se) ** 2 / 64.0
            assert r <= max(tol, 4.0 * se), (e, key, a[key], b[key], se)
    for key in chi2:
        assert chi2[key] < 4.0, (key, chi2[key])
    print("worst mixed-vs-FP64 relative difference over the sweep:", worst, "mean squared / se^2:", chi2)
