"""The reference-side adapters (icarion_b200/adapters) driven by the
reference's own engine order on the reference's own IonEnsemble.

oracle/_ref/ref_adapters is the reference harness compiled against the
reference headers with B200IntegrationStrategy and B200CollisionHandler in
the plug points (IIntegrationStrategy::step_batch, ICollisionHandler::
handle_batch) and linked against this library.  Per step it runs the
engine's prepare, step_batch, handle_batch, finalize and t += dt; the
adapters move the state through icb_update_state, icb_set_clock, icb_push,
icb_collide and icb_download_ions.  In FP64 that must give the fused
icb_advance result bit for bit (positions, velocities, active flags)."""
from __future__ import annotations

import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
from helpers import CONFIG0_DOMAIN, config0_ensemble, config0_ions, domain_json, ensemble_from_golden, golden_state
from icarion_b200 import _capi as capi
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu

BINARY = orc.HERE / "_ref" / "ref_adapters"


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert device_count() > 0, "these tests need a CUDA device"
    assert BINARY.exists(), "oracle/_ref/ref_adapters is built by make -C oracle REF=<reference tree>"


def run_adapters(st, domain: dict, steps: int, integrator: str, collision: str, dt: float, sigma: float) -> dict:
    state = {k: np.array(getattr(st, k), dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "mass",
                                                                     "charge")}
    state["ccs"] = np.full(st.n, sigma)
    state["active"] = np.asarray(st.active, dtype=np.float64)
    with tempfile.TemporaryDirectory() as td:
        ip, op = Path(td) / "in.bin", Path(td) / "out.bin"
        orc.write_state(ip, state)
        args = [str(BINARY), "adapters", f"in={ip}", f"out={op}", f"steps={steps}", f"integrator={integrator}",
                f"collision={collision}", f"dt={dt!r}", "seed=123", "precision=0"]
        args += [f"{k}={v}" for k, v in domain.items()]
        r = subprocess.run(args, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert '"strategy": "B200"' in r.stdout
        return orc.read_state(op)


def fused(st, e: dict, steps: int, integrator: int, collision: int):
    with Simulation([e], precision=capi.PREC_FP64, integrator=integrator, collision=collision, rng_seed=123) as sim:
        sim.upload(st)
        sim.advance(steps)
        return sim.download()


def same(out: dict, ref) -> None:
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(out[k], getattr(ref, k)), k
    assert np.array_equal(out["active"].astype(np.uint8), ref.active)


def test_adapters_boris_hss_equal_fused_advance():
    """Config-0 physics (Boris + HSS, 20 Td), 2,048 ions x 300 steps."""
    st0 = config0_ions(2048)
    out = run_adapters(st0, CONFIG0_DOMAIN, 300, "boris", "hss", 5e-10, 150e-20)
    same(out, fused(st0, config0_ensemble(), 300, capi.INTEGRATOR_BORIS, capi.COLLISION_HSS))


def test_adapters_rk4_fticr_equal_fused_advance(golden):
    """RK4 in the FT-ICR trap at 7 T (B through the integrator), collision free."""
    import json
    z = golden("push_rk4_fticr.npz")
    st0 = golden_state(z)
    out = run_adapters(st0, json.loads(str(z["domain"])), 500, "rk4", "none", float(z["dt"]), 150e-20)
    same(out, fused(st0, ensemble_from_golden(z), 500, capi.INTEGRATOR_RK4, capi.COLLISION_NONE))
