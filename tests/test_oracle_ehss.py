"""EHSS scattering (CPU): the oracle's restatement with Philox against the
reference's own CollisionKernels::ehss_collision (compiled harness) on the
same molecule and collision inputs — the distribution of the deflection
cosine (two-sample KS, p > 0.001) and the mean momentum transfer (within 4
standard errors) agree; energy and momentum are conserved per collision."""
from __future__ import annotations

import numpy as np
import pytest
from scipy import stats

import oracle as orc

AMU = 1.66053906660e-27


def molecule():
    """A bent 7-atom chain (C-like spheres of 1.7 A), about 6 A long."""
    xs = np.array([[-3.0, 0.0, 0.0], [-2.0, 0.8, 0.0], [-1.0, 0.0, 0.3], [0.0, 0.9, 0.0],
                   [1.0, 0.0, -0.3], [2.0, 0.8, 0.0], [3.0, 0.0, 0.0]]) * 1e-10
    return np.column_stack([xs, np.full(7, 1.7e-10)])


@pytest.mark.skipif(not orc.HARNESS.exists(), reason="compiled reference harness not built")
def test_ehss_law_matches_reference_kernel():
    n = 20000
    rng = np.random.default_rng(2)
    vi = np.tile([300.0, -100.0, 800.0], (n, 1)) + rng.normal(0, 50.0, (n, 3))
    vn = rng.normal(0, 300.0, (n, 3))
    mi, mn, rg = 300 * AMU, 28.0134 * AMU, 1.8e-10
    at = molecule()
    ref = orc.harness_ehss(at, rg, vi, vn, mi, mn, seed=9)
    orc.set_ehss(at, rg)
    mine = orc.ehss_scatter_many(vi, vn, mi, mn, seed=9)

    def cos_defl(out):
        vcom = (vi * mi + vn * mn) / (mi + mn)
        g0 = vi - vn
        g1 = (out - vcom) * (mi + mn) / mn
        return np.sum(g0 * g1, axis=1) / (np.linalg.norm(g0, axis=1) * np.linalg.norm(g1, axis=1))

    c_ref, c_me = cos_defl(ref), cos_defl(mine)
    assert stats.ks_2samp(c_ref, c_me).pvalue > 1e-3
    dp_ref = mi * (ref - vi)
    dp_me = mi * (mine - vi)
    se = np.hypot(dp_ref.std(axis=0), dp_me.std(axis=0)) / np.sqrt(n)
    assert np.all(np.abs(dp_ref.mean(axis=0) - dp_me.mean(axis=0)) <= 4 * se)
    # elastic: |g| and the centre-of-mass velocity are conserved
    vcom0 = (vi * mi + vn * mn) / (mi + mn)
    g1 = (mine - vcom0) * (mi + mn) / mn
    np.testing.assert_allclose(np.linalg.norm(g1, axis=1), np.linalg.norm(vi - vn, axis=1), rtol=1e-12)
