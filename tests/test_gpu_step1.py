"""The per-step kernel (icb_config.collision_test = ICB_TEST_PER_STEP): one
engine step per launch with the stateless collision test.

Tolerances (stated per test):
  * FP64 against the oracle's stateless mode (collision 8) with the same
    Philox streams: >= 99 % of ions to 1e-9 relative, collision counts within
    0.5 %, death and arrival times within 1e-9 relative for >= 98 % of
    the ions where both recorded them (an ion whose trajectory differs in
    its last bits, e.g. after one collision whose sampled velocity rounds
    differently, crosses the plane at a time that differs in its last
    bits too);
  * results independent of steps per launch (FP64, bit for bit);
  * collision free: bit-identical to the reference's own Boris push;
  * mixed against FP64: mean drift within 4 standard errors, collision count
    within 1 %.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from helpers import config0_ensemble, config0_ions, ensemble_from_golden, golden_state, oracle_state
from icarion_b200 import _capi as capi
from icarion_b200._capi import IcbError
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu
KEYS = ("x", "y", "z", "vx", "vy", "vz")


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def step1(st0, e, steps, precision=capi.PREC_FP64, chunks=None, n_ens=1, **kw):
    with Simulation([e] * n_ens, precision=precision, collision=kw.pop("collision", capi.COLLISION_HSS),
                    rng_seed=123, collision_test=capi.TEST_PER_STEP, **kw) as sim:
        n = st0.x.shape[0]
        sim.upload(st0, ens_offsets=None if n_ens == 1 else (np.arange(n_ens + 1) * (n // n_ens)))
        tot = {"collisions": 0, "candidates": 0}
        for k in (chunks or [steps]):
            rs = sim.advance(k)
            for key in tot:
                tot[key] += rs[key]
        return sim.download(), tot


def test_fp64_per_step_kernel_matches_oracle():
    """Config-0 physics with a small cylinder (deaths) and a detector plane
    at 0.3 mm (arrivals), 2,048 ions x 2,000 steps."""
    e = config0_ensemble(detector_z_m=3e-4)
    e.update(radius_m=1.2e-3, length_m=4e-3, origin_m=[0.0, 0.0, -2e-3])
    st0 = config0_ions(2048)
    out, tot = step1(st0, e, 2000)
    ost = oracle_state(st0)
    r = orc.run(e, ost, 2000, integrator=0, collision=8, seed=123)
    live = (out.active != 0) & (ost["active"] != 0)
    pos = np.stack([getattr(out, k) for k in KEYS[:3]])[:, live]
    opos = np.stack([ost[k] for k in KEYS[:3]])[:, live]
    vel = np.stack([getattr(out, k) for k in KEYS[3:]])[:, live]
    ovel = np.stack([ost[k] for k in KEYS[3:]])[:, live]
    rel = np.maximum(np.linalg.norm(pos - opos, axis=0) / np.linalg.norm(opos, axis=0),
                     np.linalg.norm(vel - ovel, axis=0) / np.linalg.norm(ovel, axis=0))
    assert float(np.mean(rel < 1e-9)) >= 0.99, np.sort(rel)[-5:]
    assert abs(tot["collisions"] - r["collisions"]) <= 0.005 * r["collisions"]
    assert r["collisions"] > 0.05 * 2048 * 2000
    dead = (out.active == 0) & (ost["active"] == 0)
    # relative to the time, or to one step for ions removed at t = 0
    scale_d = np.maximum(ost["t_death"][dead], e["dt_s"])
    rel_death = np.abs(out.t_death[dead] - ost["t_death"][dead]) / scale_d
    assert dead.sum() > 100 and np.mean(rel_death <= 1e-9) >= 0.98, np.sort(rel_death)[-5:]
    arr = (out.t_arrival >= 0) & (ost["t_arrival"] >= 0)
    rel_arr = np.abs(out.t_arrival[arr] - ost["t_arrival"][arr]) / np.maximum(ost["t_arrival"][arr], e["dt_s"])
    print("exact arrival times:", float(np.mean(rel_arr == 0.0)), "within 1e-9:", float(np.mean(rel_arr <= 1e-9)))
    assert arr.sum() > 100 and np.mean(rel_arr <= 1e-9) >= 0.98, np.sort(rel_arr)[-5:]


def test_per_step_kernel_results_do_not_depend_on_steps_per_launch():
    e = config0_ensemble()
    st0 = config0_ions(3000)
    a, ta = step1(st0, e, 600)                                   # one step per launch
    b, tb = step1(st0, e, 600, steps_per_launch=16, chunks=[250, 250, 100])
    for k in KEYS + ("active",):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert ta == tb


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED, capi.PREC_MIXED_HILO])
def test_per_step_kernel_tiles_across_ensembles_and_launch_chunks(precision):
    """70 ensembles of 37 ions with the same physics against one ensemble of
    the same 2,590 ions: bit-identical (the ion id, not the ensemble, keys
    the random numbers).  The ensembles run in two launch chunks (64 per
    launch), the second starting at ion 2,368, inside a 256-ion tile, so
    tiles loaded by bulk copies and tiles cut by a chunk's ends (loaded per
    thread) both take part, as does the per-ion ensemble search."""
    e = config0_ensemble(detector_z_m=3e-4)
    e.update(radius_m=1.2e-3, length_m=4e-3, origin_m=[0.0, 0.0, -2e-3])
    st0 = config0_ions(70 * 37)
    a, ta = step1(st0, e, 300, precision=precision)
    b, tb = step1(st0, e, 300, precision=precision, n_ens=70)
    for k in KEYS + ("active", "t_death", "t_arrival"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert ta == tb and ta["collisions"] > 0


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_ions_moved_outside_between_steps_are_removed_at_the_next_prepare(precision):
    """Once a step has finalized every ion the kernel skips the next step's
    domain test at prepare; state written by the host (icb_update_state)
    brings it back: ions moved outside the cylinder between two steps die at
    the next step's start time, the others step on."""
    e = config0_ensemble(detector_z_m=1e30)
    e.update(radius_m=1.2e-3, length_m=4e-3, origin_m=[0.0, 0.0, -2e-3])
    st0 = config0_ions(1000)
    st0.x[:] *= 0.2
    st0.y[:] *= 0.2
    st0.z[:] *= 0.2
    with Simulation([e], precision=precision, collision=capi.COLLISION_HSS, rng_seed=123,
                    collision_test=capi.TEST_PER_STEP) as sim:
        sim.upload(st0)
        for _ in range(3):
            sim.advance(1)
        st = sim.download()
        assert int(st.active.sum()) == 1000
        moved = np.arange(0, 1000, 7)
        st.x[moved] = 5e-3                       # beyond the 1.2 mm radius
        sim.update_state(st)
        _, t_before = sim.clock()
        sim.advance(1)
        out = sim.download()
    assert np.all(out.active[moved] == 0)
    assert np.all(out.t_death[moved] == t_before[0])
    keep = np.setdiff1d(np.arange(1000), moved)
    assert np.all(out.active[keep] == 1)
    assert np.all(out.x[moved] == 5e-3)          # removed before the push: not moved


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_per_step_advance_host_equals_separate_calls(precision):
    """icb_advance_host in per-step mode: 4 overlapped ion chunks (their
    launches cut tiles at the chunk ends and always prepare) give the state
    of update_state + advance + download (one chunk) bit for bit."""
    e = config0_ensemble(detector_z_m=3e-4)
    e.update(radius_m=1.2e-3, length_m=4e-3, origin_m=[0.0, 0.0, -2e-3])
    st0 = config0_ions(3000)
    outs = []
    for chunks in (1, 4):
        with Simulation([e], precision=precision, collision=capi.COLLISION_HSS, rng_seed=5,
                        collision_test=capi.TEST_PER_STEP) as sim:
            sim.upload(st0)
            host = st0.copy()
            host.t_death = host.t_arrival = None
            tot = 0
            for _ in range(3):
                tot += sim.advance_host(host, 50, n_chunks=chunks)["collisions"]
            outs.append((host, tot))
    for k in KEYS + ("active",):
        assert np.array_equal(getattr(outs[0][0], k), getattr(outs[1][0], k)), k
    assert outs[0][1] == outs[1][1] > 0


def test_collision_free_per_step_kernel_is_the_reference_push(golden):
    z = golden("push_boris_ims.npz")
    out, _ = step1(golden_state(z), ensemble_from_golden(z), int(z["steps"]), collision=capi.COLLISION_NONE)
    for k in KEYS:
        assert np.array_equal(getattr(out, k), z["out_" + k]), k


def test_mixed_per_step_kernel_tracks_fp64():
    e = config0_ensemble(detector_z_m=1e30)
    st0 = config0_ions(20000)
    res = {p: step1(st0, e, 2000, precision=p) for p in (capi.PREC_FP64, capi.PREC_MIXED, capi.PREC_MIXED_HILO)}
    dz64 = res[capi.PREC_FP64][0].z - st0.z
    for p in (capi.PREC_MIXED, capi.PREC_MIXED_HILO):
        dz = res[p][0].z - st0.z
        assert abs(dz.mean() - dz64.mean()) <= 4 * dz64.std() / np.sqrt(dz64.size), p
        assert abs(res[p][1]["collisions"] / res[capi.PREC_FP64][1]["collisions"] - 1.0) < 0.01, p


def test_per_ion_species_path():
    """Ions of different masses in one ensemble: the kernel reads the per-ion
    mass and charge (FP64 vs oracle)."""
    e = config0_ensemble(detector_z_m=1e30)
    st0 = config0_ions(1024)
    st0.mass[::2] *= 1.5
    out, tot = step1(st0, e, 1000)
    ost = oracle_state(st0)
    r = orc.run(e, ost, 1000, integrator=0, collision=8, seed=123)
    rel = np.abs(out.z - ost["z"]) / np.abs(ost["z"])
    assert float(np.mean(rel < 1e-9)) >= 0.99
    assert abs(tot["collisions"] - r["collisions"]) <= 0.005 * r["collisions"]


def test_per_step_kernel_rejects_what_it_does_not_run():
    e = config0_ensemble()
    with pytest.raises(IcbError) as ei:
        Simulation([e], integrator=capi.INTEGRATOR_RK4, collision_test=capi.TEST_PER_STEP)
    assert ei.value.code == capi.ICB_ERR_UNSUPPORTED
    with Simulation([e], precision=capi.PREC_FP64, collision_test=capi.TEST_PER_STEP) as sim:
        st = config0_ions(64)
        st.birth = np.zeros(64)
        with pytest.raises(IcbError):
            sim.upload(st)
        sim.upload(config0_ions(64))
        with pytest.raises(IcbError):
            sim.step_batch()                 # unfused plug points use the clock kernels
        with pytest.raises(IcbError):
            sim.autotune(100)
        sim.advance(10)
