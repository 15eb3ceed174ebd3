"""Event-to-event drift of the float forms against their step-by-step loop.

Both float stepping modes draw the same Philox counters at the same steps,
so an ion follows the same history in both until float rounding flips a
decision (rare).  The FP64 form draws its uniforms at full 32-bit resolution
(and angles over (0, 2 pi)), so with collisions it is a per-ion reference
only until the first one; without collisions it is exact.  Tolerances are
stated per test.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import config0_ensemble, config0_ions
from icarion_b200 import _capi as capi
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu
DT = 5e-10


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def _run(e, st0, steps, precision, stepping, collision=capi.COLLISION_HSS, **kw):
    with Simulation([e], precision=precision, collision=collision, rng_seed=77, stepping=stepping, **kw) as sim:
        sim.upload(st0)
        rs = sim.advance(steps)
        return sim.download(), rs


def _rel_err(a, b):
    """Per-ion max of the relative position and velocity errors of a vs b."""
    pa = np.stack([a.x, a.y, a.z])
    pb = np.stack([b.x, b.y, b.z])
    va = np.stack([a.vx, a.vy, a.vz])
    vb = np.stack([b.vx, b.vy, b.vz])
    rp = np.linalg.norm(pa - pb, axis=0) / np.maximum(np.linalg.norm(pb, axis=0), 1e-6)
    rv = np.linalg.norm(va - vb, axis=0) / np.maximum(np.linalg.norm(vb, axis=0), 1e-3)
    return np.maximum(rp, rv)


@pytest.mark.parametrize("precision", [capi.PREC_MIXED, capi.PREC_MIXED_HILO])
@pytest.mark.parametrize("collision", [capi.COLLISION_HSS, capi.COLLISION_LANGEVIN])
def test_event_drift_follows_step_by_step(precision, collision):
    """With collisions: the same events and counts as the step-by-step float
    loop; positions and velocities within 1e-4 for >= 98 % of ions (the loop's
    own v += a dt/2 rounding reaches 1e-5 over long collision-free runs)."""
    e = config0_ensemble()
    st0 = config0_ions(4096)
    ev, rs_ev = _run(e, st0, 3000, precision, capi.STEPPING_EVENTS, collision)
    ps, rs_ps = _run(e, st0, 3000, precision, capi.STEPPING_PER_STEP, collision)
    ok = _rel_err(ev, ps) <= 1e-4
    assert ok.mean() >= 0.98, ok.mean()
    for key in ("candidates", "collisions"):
        assert abs(rs_ev[key] - rs_ps[key]) <= 0.005 * max(rs_ps[key], 1), (key, rs_ev[key], rs_ps[key])
    assert int(ev.active.sum()) == int(ps.active.sum()) == 4096


def _death_step(st):
    """Step index of the death time (FP64 sums t += dt like the reference,
    the float forms take t0 + k dt: the same step, rounded differently)."""
    return np.where(st.active == 0, np.rint(st.t_death / DT), -1)


def _cylinder(detector_z_m=4e-4):
    """2.6 mm x 0.6 mm cylinder with the config-0 axial voltage: 186 kV/m."""
    e = config0_ensemble(detector_z_m=detector_z_m, dt=DT)
    e.update(radius_m=6e-4, length_m=2.6e-3, origin_m=[0.0, 0.0, -1.3e-3])
    return e


@pytest.mark.parametrize("precision", [capi.PREC_MIXED, capi.PREC_MIXED_HILO])
def test_collision_free_drift_exits_and_arrivals_match_fp64(precision):
    """Without collisions the FP64 step-by-step run is an exact per-ion
    reference (the oracle's arithmetic).  Event drift: positions and
    velocities within 1e-5, the same death step for >= 99 % of ions, first
    detector crossings within 1e-3 dt, and no larger errors than the
    step-by-step float loop."""
    e = _cylinder()
    st0 = config0_ions(4096)
    ref, _ = _run(e, st0, 2000, capi.PREC_FP64, capi.STEPPING_PER_STEP, capi.COLLISION_NONE)
    ev, rs_ev = _run(e, st0, 2000, precision, capi.STEPPING_EVENTS, capi.COLLISION_NONE)
    ps, _ = _run(e, st0, 2000, precision, capi.STEPPING_PER_STEP, capi.COLLISION_NONE)
    assert (ref.active == 0).sum() > 4096 // 2
    same = (ev.active == ref.active) & (_death_step(ev) == _death_step(ref))
    assert same.mean() >= 0.99, same.mean()
    err_ev, err_ps = _rel_err(ev, ref), _rel_err(ps, ref)
    assert np.mean(err_ev <= 1e-5) >= 0.99
    assert np.median(err_ev) <= np.median(err_ps) + 1e-12, (np.median(err_ev), np.median(err_ps))
    arr = ref.t_arrival >= 0
    assert arr.sum() > 500 and np.mean((ev.t_arrival >= 0) == arr) >= 0.999
    arr &= ev.t_arrival >= 0
    d_ev = np.abs(ev.t_arrival[arr] - ref.t_arrival[arr])
    d_ps = np.abs(ps.t_arrival[arr] - ref.t_arrival[arr])
    assert np.mean(d_ev <= 1e-3 * DT) >= 0.99, np.quantile(d_ev / DT, [0.5, 0.99, 1])
    assert np.median(d_ev) <= np.median(d_ps) + 1e-18
    assert rs_ev["deaths"] == int(np.sum(ev.active == 0))
    assert rs_ev["arrivals"] == int(np.sum(ev.t_arrival >= 0))


def test_event_drift_exits_and_arrivals_follow_step_by_step():
    """With collisions in the strong-field cylinder: the same death steps as
    the step-by-step float loop for >= 98 % of ions and first crossings within
    2e-2 dt (that loop's own rounding moves them by up to ~7e-3 dt)."""
    e = _cylinder()
    st0 = config0_ions(4096)
    ev, rs_ev = _run(e, st0, 4000, capi.PREC_MIXED, capi.STEPPING_EVENTS)
    ps, _ = _run(e, st0, 4000, capi.PREC_MIXED, capi.STEPPING_PER_STEP)
    assert (ps.active == 0).sum() > 4096 // 4
    same = (ev.active == ps.active) & (ev.t_death == ps.t_death)
    assert same.mean() >= 0.98, same.mean()
    arr_ps, arr_ev = ps.t_arrival >= 0, ev.t_arrival >= 0
    assert arr_ps.sum() > 200
    both = arr_ps & arr_ev
    assert both.sum() >= 0.98 * max(arr_ps.sum(), arr_ev.sum())
    close = np.abs(ev.t_arrival[both] - ps.t_arrival[both]) <= 2e-2 * DT
    assert close.mean() >= 0.98, close.mean()
    assert rs_ev["deaths"] == int(np.sum(ev.active == 0))
    assert rs_ev["arrivals"] == int(arr_ev.sum())


def test_short_launches_check_every_step():
    e = _cylinder()
    st0 = config0_ions(2048)
    ref, _ = _run(e, st0, 1500, capi.PREC_FP64, capi.STEPPING_PER_STEP, capi.COLLISION_NONE, steps_per_launch=5)
    ev, _ = _run(e, st0, 1500, capi.PREC_MIXED, capi.STEPPING_EVENTS, capi.COLLISION_NONE, steps_per_launch=5)
    same = (ev.active == ref.active) & (_death_step(ev) == _death_step(ref))
    assert (ref.active == 0).sum() > 2048 // 2
    assert same.mean() >= 0.99, same.mean()
    assert np.mean(_rel_err(ev, ref) <= 1e-5) >= 0.99


def test_every_ion_of_a_large_cloud_is_advanced():
    """300,000 ions (about 2.6 waves of resident blocks): every ion moves, and
    the event form follows the step-by-step loop."""
    e = config0_ensemble()
    st0 = config0_ions(300_000)
    ev, rs_ev = _run(e, st0, 400, capi.PREC_MIXED, capi.STEPPING_EVENTS)
    ps, rs_ps = _run(e, st0, 400, capi.PREC_MIXED, capi.STEPPING_PER_STEP)
    assert np.all(ev.z != st0.z) and np.all(ev.vz != st0.vz)
    assert np.mean(_rel_err(ev, ps) <= 1e-4) >= 0.98
    assert abs(rs_ev["collisions"] - rs_ps["collisions"]) <= 0.005 * rs_ps["collisions"]
    assert int(ev.active.sum()) == int(ps.active.sum())


def test_births_follow_step_by_step():
    """Unborn ions wait unmoved until the first step whose start time reaches
    their birth time, then step (a warp with an unborn ion takes the
    step-by-step loop in both stepping modes)."""
    e = config0_ensemble()
    n = 4096
    st = config0_ions(n)
    rng = np.random.default_rng(5)
    st.birth = rng.uniform(0.0, 1100 * DT, n)
    st.birth[:64] = 1.0                     # never born within the run
    st.birth[64:128] = 0.0
    st.birth[128:192] = 700 * DT            # exactly on a step start
    outs = []
    for stepping in (capi.STEPPING_EVENTS, capi.STEPPING_PER_STEP):
        with Simulation([e], precision=capi.PREC_MIXED, collision=capi.COLLISION_HSS, rng_seed=77,
                        stepping=stepping, steps_per_launch=400) as sim:
            sim.upload(st)
            sim.advance(500)
            mid = sim.download()
            sim.advance(700)
            outs.append((mid, sim.download()))
    (mid_ev, ev), (mid_ps, ps) = outs
    for a, b in ((mid_ev, mid_ps), (ev, ps)):
        assert np.array_equal(a.active, b.active)
        unborn = b.active == 0
        assert np.array_equal(a.z[unborn], st.z[unborn]) and np.array_equal(b.z[unborn], st.z[unborn])
        assert np.mean(_rel_err(a, b) <= 1e-4) >= 0.98
    assert not ev.active[:64].any() and ev.active[64:].all()


def test_stepping_mode_is_validated():
    with pytest.raises(capi.IcbError):
        Simulation([config0_ensemble()], stepping=7)
