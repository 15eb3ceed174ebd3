"""Batched ensembles (the E/N sweep) on the device: one handle advancing
many ensembles with different fields, species and dt gives, per ensemble,
exactly the result of running that ensemble alone with the same ion ids
(FP64, bit for bit), across the 64-ensembles-per-launch chunk boundary."""
from __future__ import annotations

import numpy as np
import pytest

from icarion_b200 import _capi as capi
from icarion_b200 import sweep
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu
KEYS = ("x", "y", "z", "vx", "vy", "vz", "active", "t_death", "t_arrival")


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def _run(ensembles, st, offsets, first_id, steps, precision, **kw):
    with Simulation(ensembles, precision=precision, integrator=capi.INTEGRATOR_BORIS,
                    collision=capi.COLLISION_HSS, rng_seed=99, **kw) as sim:
        sim.upload(st, ens_offsets=offsets, first_id=first_id)
        rs = sim.advance(steps)
        return sim.download(), sim.clock(), rs


def test_batched_sweep_equals_separate_runs_fp64():
    rng = np.random.default_rng(5)
    counts = rng.integers(20, 300, size=66)
    sw = sweep.en_sweep(n_ensembles=66, counts=counts)
    steps = 700
    out, (step, t), rs = _run(sw.ensembles, sw.ions, sw.offsets, 0, steps, capi.PREC_FP64, steps_per_launch=256)
    assert step == steps and rs["collisions"] > 0
    dts = np.array([e["dt_s"] for e in sw.ensembles])
    np.testing.assert_allclose(t, steps * dts, rtol=1e-12)
    for e in (0, 1, 40, 63, 64, 65):
        lo, hi = int(sw.offsets[e]), int(sw.offsets[e + 1])
        alone, (s1, t1), _ = _run([sw.ensembles[e]], sweep.subset(sw.ions, lo, hi), None, lo, steps,
                                  capi.PREC_FP64, steps_per_launch=333)
        assert s1 == steps and t1[0] == t[e]
        for k in KEYS:
            assert np.array_equal(getattr(alone, k), getattr(out, k)[lo:hi]), (e, k)


def test_batched_sweep_mixed_tracks_fp64_drift():
    """Mixed precision on the batched sweep: per-ensemble mean z displacement
    after 2000 steps agrees with FP64 within 4 standard errors plus 1e-3
    relative (the ions' Philox streams are the same in both forms)."""
    counts = np.full(12, 6000)
    sw = sweep.en_sweep(n_ensembles=12, counts=counts)
    steps = 2000
    f64, _, _ = _run(sw.ensembles, sw.ions, sw.offsets, 0, steps, capi.PREC_FP64)
    mix, _, _ = _run(sw.ensembles, sw.ions, sw.offsets, 0, steps, capi.PREC_MIXED)
    for e in range(12):
        lo, hi = int(sw.offsets[e]), int(sw.offsets[e + 1])
        dz64 = f64.z[lo:hi] - sw.ions.z[lo:hi]
        dzm = mix.z[lo:hi] - sw.ions.z[lo:hi]
        se = np.std(dz64) / np.sqrt(hi - lo)
        assert abs(dzm.mean() - dz64.mean()) <= 4 * se + 1e-3 * abs(dz64.mean()), e
