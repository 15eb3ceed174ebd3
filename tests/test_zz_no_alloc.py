"""icb_moments_noalloc: moments of caller-owned device arrays with no device
allocation inside the library (for callers whose device memory is all
reserved by their own allocator, or who run under a fixed device-memory
budget).  Checked against icb_moments (the handle-based entry point) on two
calls in a row, within the moment tolerance used elsewhere (rtol 1e-12).

Collected last (file name) so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from helpers import config0_ensemble, config0_ions
from icarion_b200 import _capi as capi
from icarion_b200.sim import Simulation, device_count

pytestmark = pytest.mark.gpu


def _dev(a: np.ndarray):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _noalloc(st, ref, out):
    import torch
    arrays = [_dev(getattr(st, k)) for k in ("x", "y", "z", "vx", "vy", "vz")]
    refs = [_dev(r) for r in ref]
    act = _dev(st.active)
    ta, td = _dev(st.t_arrival), _dev(st.t_death)
    torch.cuda.synchronize()
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    rc = capi.lib().icb_moments_noalloc(0, st.n, *[ptr(t) for t in arrays], *[ptr(t) for t in refs], ptr(act),
                                        ptr(ta), ptr(td), ptr(out), None)
    capi.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy().copy()


def test_noalloc_moments_match_handle_moments_on_two_calls():
    import torch
    assert device_count() > 0
    n = 20000
    e = config0_ensemble(detector_z_m=2.0e-4)
    st0 = config0_ions(n)
    ref = (st0.x.copy(), st0.y.copy(), st0.z.copy())   # the handle's reference = upload positions
    out = torch.zeros(capi.N_MOMENTS, dtype=torch.float64, device="cuda")
    with Simulation([e], precision=capi.PREC_MIXED, collision=capi.COLLISION_HSS, rng_seed=7) as sim:
        sim.upload(st0)
        for _ in range(2):
            sim.advance(500)
            want = sim.moments()[0]
            got = _noalloc(sim.download(), ref, out)
            np.testing.assert_allclose(got, want, rtol=1e-12, atol=0.0)
            assert want[0] > 0 and want[11] > 0        # active ions and detector arrivals present


def test_noalloc_rejects_more_ions_than_its_scratch_holds():
    import torch
    assert device_count() > 0
    small = torch.zeros(8, dtype=torch.float64, device="cuda")
    flags = torch.zeros(8, dtype=torch.uint8, device="cuda")
    p = C.c_void_p(small.data_ptr())
    rc = capi.lib().icb_moments_noalloc(0, 33_554_433, p, p, p, p, p, p, p, p, p, C.c_void_p(flags.data_ptr()),
                                        None, None, p, None)
    assert rc == capi.ICB_ERR_INVALID_ARGUMENT
    assert b"33554432" in capi.lib().icb_last_error()
