"""Space charge on the device (icb_spacecharge_configure / _field) against
the numpy oracle of both solvers, the reference's own two-ion GPU test, and
a pushed two-ion system (momentum and energy).

Tolerances: the isolated P3M field equals the oracle's to 1e-6 of the
cloud's RMS field (the particle-particle term is interpolated from a
4,096-interval table of the long-range kernel, ~3e-8 relative; FFT and
summation order add rounding only); the reference periodic solver's float
output to 1e-6 of its largest field."""
from __future__ import annotations

import numpy as np
import pytest

import p3m
from icarion_b200 import _capi as capi
from icarion_b200 import config as cfg
from icarion_b200.sim import IonState, Simulation, device_count

pytestmark = pytest.mark.gpu
E_CHARGE = 1.602176634e-19
AMU = 1.66053906660e-27


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"


def _state(x, y, z, q, active=None, mass_da=100.0, v=None):
    n = x.shape[0]
    st = IonState.empty(n)
    st.x[:], st.y[:], st.z[:] = x, y, z
    if v is not None:
        st.vx[:], st.vy[:], st.vz[:] = v
    st.mass[:] = mass_da * AMU
    st.charge[:] = q
    if active is not None:
        st.active[:] = active
    return st


def _field_free(dt=5e-10):
    # no external field; large cylinder around the origin; N2 at 300 K, 1000 Pa
    domain = {"instrument": "IMS", "geometry": {"origin_m": [0.0, 0.0, -0.05], "length_m": 0.1, "radius_m": 0.05},
              "env": {"temperature_K": 300.0, "pressure_Pa": 1000.0, "gas_species": "N2"},
              "fields": {"DC": {"EN_Td": 0.0}}}
    return cfg.ensemble_params(domain, 150e-20, dt)


def _sim(st, precision=capi.PREC_FP64, **kw):
    sim = Simulation([_field_free()], precision=precision, collision=capi.COLLISION_NONE, rng_seed=1, **kw)
    sim.upload(st)
    return sim


def _cloud(n, seed=1, sigma=1e-3):
    rng = np.random.default_rng(seed)
    x, y, z = rng.normal(0.0, sigma, (3, n))
    q = np.full(n, E_CHARGE)
    q[::9] = -E_CHARGE
    return x, y, z, q


@pytest.mark.parametrize("precision,tol", [(capi.PREC_FP64, 1e-6), (capi.PREC_MIXED, 1e-4)])
def test_isolated_p3m_matches_oracle(precision, tol):
    """FP64: the particle-particle sums in FP64 (tolerance 1e-6 of the RMS
    field from the kernel table); mixed: in float on positions relative to
    the mesh origin (1e-4)."""
    x, y, z, q = _cloud(3000)
    act = np.ones(3000, dtype=np.uint8)
    act[::13] = 0
    n = (32, 32, 32)
    lo, hi = np.full(3, -6e-3), np.full(3, 6e-3)
    h = (hi - lo) / 32
    want = p3m.p3m_field(x, y, z, q, act, lo, h, n, 1.0 / h.max(), 2.0 * h.max())
    with _sim(_state(x, y, z, q, act), precision=precision) as sim:
        sim.configure_space_charge(capi.SC_P3M_ISOLATED, n, lo, hi)
        got = sim.space_charge_field()
        again = sim.space_charge_field()
    assert np.array_equal(got, again)                      # deterministic (no atomics)
    rms = np.sqrt(np.mean(np.sum(want ** 2, axis=0)))
    assert np.max(np.abs(got - want)) <= tol * rms
    assert np.all(got[:, act == 0] == 0.0)


@pytest.mark.parametrize("precision,tol", [(capi.PREC_FP64, 1e-6), (capi.PREC_MIXED, 1e-4)])
def test_box_mesh_matches_oracle_and_solves_keep_no_state(precision, tol):
    """A mesh with three different sizes (the mixed form's single-precision
    mesh: 2D (y, z) transforms of the mesh planes, 1D x transforms of the
    spectrum, folded kernel quadrant).  The field is within `tol` of the
    oracle's RMS field (as on the cubic mesh), and a solve after another
    cloud equals a fresh solver's solve bit for bit (nothing of the first
    cloud stays in the grids' padding or the spectrum's upper planes)."""
    n = (32, 24, 20)
    lo, hi = np.array([-6e-3, -5e-3, -4.5e-3]), np.array([6e-3, 5e-3, 4.5e-3])
    h = (hi - lo) / np.array(n)
    first = _cloud(3000, seed=3, sigma=0.8e-3)
    x, y, z, q = _cloud(3000)
    act = np.ones(3000, dtype=np.uint8)
    want = p3m.p3m_field(x, y, z, q, act, lo, h, n, 1.0 / h.max(), 2.0 * h.max())
    with _sim(_state(*first), precision=precision) as sim:
        sim.configure_space_charge(capi.SC_P3M_ISOLATED, n, lo, hi)
        sim.space_charge_field()
        sim.upload(_state(x, y, z, q))
        got = sim.space_charge_field()
    with _sim(_state(x, y, z, q), precision=precision) as sim:
        sim.configure_space_charge(capi.SC_P3M_ISOLATED, n, lo, hi)
        fresh = sim.space_charge_field()
    assert np.array_equal(got, fresh)
    rms = np.sqrt(np.mean(np.sum(want ** 2, axis=0)))
    assert np.max(np.abs(got - want)) <= tol * rms


def test_fused_x_pass_mesh_matches_oracle():
    """A 128-node x axis (padded x length 256) runs the fused x pass:
    forward transform, the three kernel products and the inverse transforms
    per spectrum column in one kernel.  On a 128 x 25 x 20 mesh (a column
    count that is no multiple of the kernel's 16 columns per block), with
    the particle-particle cutoff at 1/100 cell so that the mesh part alone
    is compared, the mixed form's field is within 1e-5 of the oracle's RMS
    field (float transforms), and a solve after another cloud equals a
    fresh solver's bit for bit."""
    n = (128, 25, 20)
    h = 1e-4
    lo = np.array([-64 * h, -12.5 * h, -10 * h])
    hi = -lo
    first = _cloud(3000, seed=5, sigma=2e-4)
    x, y, z, q = _cloud(3000, seed=7, sigma=2.5e-4)
    act = np.ones(3000, dtype=np.uint8)
    hs = (hi - lo) / np.array(n)
    want = p3m.p3m_field(x, y, z, q, act, lo, hs, n, 1.0 / hs.max(), 0.01 * hs.max())
    kw = dict(pp_cutoff_cells=0.01)
    with _sim(_state(*first), precision=capi.PREC_MIXED) as sim:
        sim.configure_space_charge(capi.SC_P3M_ISOLATED, n, lo, hi, **kw)
        sim.space_charge_field()
        sim.upload(_state(x, y, z, q))
        got = sim.space_charge_field()
    with _sim(_state(x, y, z, q), precision=capi.PREC_MIXED) as sim:
        sim.configure_space_charge(capi.SC_P3M_ISOLATED, n, lo, hi, **kw)
        fresh = sim.space_charge_field()
    assert np.array_equal(got, fresh)
    inside = np.any(want != 0.0, axis=0)
    assert inside.sum() > 2000
    rms = np.sqrt(np.mean(np.sum(want[:, inside] ** 2, axis=0)))
    err = float(np.max(np.abs(got - want)))
    print("fused x pass: max error / RMS field", err / rms)
    assert err <= 1e-5 * rms


def test_reference_periodic_solver_matches_oracle():
    x, y, z, q = _cloud(2000, seed=2)
    act = np.zeros(2000, dtype=np.uint8)                  # the reference solver ignores activity
    n = (32, 24, 20)
    lo, hi = [-5e-3, -4e-3, -3.5e-3], [5e-3, 4e-3, 3.5e-3]
    want = p3m.periodic_pm_field(x, y, z, q, lo, hi, n)
    with _sim(_state(x, y, z, q, act)) as sim:
        sim.configure_space_charge(capi.SC_PM_PERIODIC_REF, n, lo, hi, field_bound=1.0)
        got = sim.space_charge_field()
    assert np.max(np.abs(got - want)) <= 1e-6 * np.max(np.abs(want))


@pytest.mark.skipif(not p3m.REF_P3M.exists(), reason="reference GPU solver not built (oracle/Makefile)")
def test_periodic_solver_matches_reference_gpu_code():
    """The library's ICB_SC_PM_PERIODIC_REF and the numpy restatement against
    the reference's own GPUSpaceChargeP3M run on the same ions: within 1e-5
    of the largest field (float weights and outputs on both sides; the
    reference deposits with atomics, in no fixed order)."""
    x, y, z, q = _cloud(2000, seed=2)
    n = (32, 24, 20)
    lo, hi = [-5e-3, -4e-3, -3.5e-3], [5e-3, 4e-3, 3.5e-3]
    ref = p3m.periodic_pm_field_reference_gpu(x, y, z, q, lo, hi, n)
    want = p3m.periodic_pm_field(x, y, z, q, lo, hi, n)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(want - ref)) <= 1e-5 * scale
    with _sim(_state(x, y, z, q, np.zeros(2000, dtype=np.uint8))) as sim:
        sim.configure_space_charge(capi.SC_PM_PERIODIC_REF, n, lo, hi, field_bound=1.0)
        got = sim.space_charge_field()
    assert np.max(np.abs(got - ref)) <= 1e-5 * scale


@pytest.mark.parametrize("mode,tol", [(capi.SC_PM_PERIODIC_REF, 0.25), (capi.SC_P3M_ISOLATED, 2e-3)])
def test_two_ion_coulomb_case(mode, tol):
    """tests/gpu/test_gpu_space_charge.cpp:76-139 (the reference's bound is 25 %)."""
    x, y, z = np.zeros(2), np.zeros(2), np.array([0.0, 1e-3])
    want = E_CHARGE / (4 * np.pi * p3m.EPSILON_0 * 1e-6)
    with _sim(_state(x, y, z, np.full(2, E_CHARGE))) as sim:
        sim.configure_space_charge(mode, (128, 128, 128), [-2e-3, -2e-3, -1e-3], [2e-3, 2e-3, 2e-3],
                                   field_bound=1.0)
        e = sim.space_charge_field()
    assert abs(np.linalg.norm(e[:, 1]) - want) / want < tol
    assert e[2, 1] > 0 and e[2, 0] < 0
    assert abs(e[2, 0] + e[2, 1]) / want < 0.15


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED])
def test_pushed_ion_pair_conserves_momentum_and_energy(precision):
    """Two +e ions (100 Da) released 200 um apart (13 mesh cells) fly apart
    under their own field: equal and opposite momenta, and kinetic energy
    = k q^2 (1/r0 - 1/r) within 1 %."""
    r0 = 200e-6
    x, y, z = np.zeros(2), np.zeros(2), np.array([-r0 / 2, r0 / 2])
    kq2 = p3m.COULOMB_CONST * E_CHARGE ** 2
    with Simulation([_field_free(dt=5e-8)], precision=precision, collision=capi.COLLISION_NONE,
                    rng_seed=1) as sim:
        sim.upload(_state(x, y, z, np.full(2, E_CHARGE)))
        sim.configure_space_charge(capi.SC_P3M_ISOLATED, (128, 128, 128), [-1e-3] * 3, [1e-3] * 3)
        rs = sim.advance(1500)
        out = sim.download()
    assert rs["spacecharge_solves_timed"] == 64 and rs["spacecharge_ms"] > 0
    vz = out.vz
    assert vz[1] > 0 > vz[0] and abs(vz[0] + vz[1]) <= 1e-4 * abs(vz[1])
    r = out.z[1] - out.z[0]
    assert r > 1.5 * r0
    ke = 0.5 * 100 * AMU * np.sum(out.vx ** 2 + out.vy ** 2 + out.vz ** 2)
    assert abs(ke / (kq2 * (1 / r0 - 1 / r)) - 1.0) < 0.01


def test_coulomb_explosion_conserves_total_momentum():
    """Mesh forces (CIC assignment = interpolation, odd kernel) and pair
    corrections are antisymmetric: a 2,000-ion cloud blown apart by its own
    charge keeps zero total momentum to rounding (FP64)."""
    x, y, z = _cloud(2000, seed=6, sigma=1e-4)[:3]
    with Simulation([_field_free(dt=1e-9)], precision=capi.PREC_FP64, collision=capi.COLLISION_NONE,
                    rng_seed=1) as sim:
        sim.upload(_state(x, y, z, np.full(2000, E_CHARGE)))
        sim.configure_space_charge(capi.SC_P3M_ISOLATED, (64, 64, 64), [-1.5e-3] * 3, [1.5e-3] * 3)
        sim.advance(600)
        out = sim.download()
    p = np.stack([out.vx, out.vy, out.vz])
    assert np.all(out.active == 1)
    assert np.linalg.norm(p.sum(axis=1)) <= 1e-9 * np.abs(p).sum()
    # the cloud expanded
    assert np.std(out.z) > 1.02 * np.std(z)


def test_space_charge_graph_replay_and_off_switch():
    x, y, z = _cloud(500, seed=4, sigma=2e-4)[:3]
    v = np.random.default_rng(5).normal(0, 300.0, (3, 500))
    st = _state(x, y, z, np.full(500, E_CHARGE), v=v)
    outs = []
    for graphs in (0, 1):
        with _sim(st, use_graphs=graphs) as sim:
            sim.configure_space_charge(capi.SC_P3M_ISOLATED, (32, 32, 32), [-2e-3] * 3, [2e-3] * 3)
            for _ in range(3):
                sim.advance(40)
            outs.append(sim.download())
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(getattr(outs[0], k), getattr(outs[1], k)), k
    # switching space charge off gives the field-free ballistic push again
    with _sim(st) as sim:
        sim.configure_space_charge(capi.SC_P3M_ISOLATED, (32, 32, 32), [-2e-3] * 3, [2e-3] * 3)
        sim.configure_space_charge(capi.SC_OFF, (8, 8, 8), [0] * 3, [1] * 3)
        sim.advance(10)
        free = sim.download()
    np.testing.assert_allclose(free.z, st.z + 10 * 5e-10 * st.vz, rtol=1e-12, atol=1e-18)


def test_space_charge_rejects_unsupported_setups():
    x, y, z, q = _cloud(10)
    with Simulation([_field_free()], precision=capi.PREC_FP64, integrator=capi.INTEGRATOR_RK4,
                    collision=capi.COLLISION_NONE) as sim:
        sim.upload(_state(x, y, z, q))
        with pytest.raises(RuntimeError, match="Boris"):
            sim.configure_space_charge(capi.SC_P3M_ISOLATED, (16, 16, 16), [-1e-2] * 3, [1e-2] * 3)
    with _sim(_state(x, y, z, q)) as sim:
        with pytest.raises(RuntimeError, match="grid_n"):
            sim.configure_space_charge(capi.SC_P3M_ISOLATED, (4, 16, 16), [-1e-2] * 3, [1e-2] * 3)
