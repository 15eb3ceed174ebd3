"""ORACLE — test infrastructure only (the checker, never the product).

numpy restatements of the space-charge field on the batch step:

* ``direct_field``    — the reference's direct summation
  (``SpaceChargeDirectModel::update_fields``, SpaceChargeDirectModel.cpp:20-66):
  E_i = sum_j k q_j / (r^2 + eps^2) * r_hat over active j != i, pairs with
  r^2 < max(eps^2 1e-4, 1e-30) skipped; k = COULOMB_CONST (utils/constants.h:20).
  Pinned against the compiled reference (``direct_field_reference``).
* ``periodic_pm_field`` — the reference's GPU particle-mesh solver
  (GPUSpaceChargeP3M.cu:36-339, GPUSpaceChargeP3M.cpp:20-183): CIC charge
  assignment with float weights onto a z-fastest grid, periodic FFT Poisson
  solve phi_hat = rho_hat / (eps0 k^2 V) with the reference's wave numbers
  (its z length is (nz/2+1) * 2 * dz), 1/N scaling, central differences
  (one-sided at the grid edges), CIC interpolation with float weights.
  Every ion deposits (the reference passes all ions, active or not); ions
  with a grid coordinate outside [0, n-1) are skipped and get E = 0.
  Pinned against the reference's own GPU code
  (``periodic_pm_field_reference_gpu``, run on a GPU).
* ``p3m_field`` — the isolated-boundary P3M solver of this library:
  CIC charges on the mesh, convolved (zero-padded FFT, Hockney-Eastwood)
  with the sampled long-range Coulomb field of a Gaussian-screened charge,
      E_long(r) = k [erf(a r) / r^2 - (2 a / sqrt(pi)) exp(-a^2 r^2) / r],
  CIC-interpolated to the ions, plus a particle-particle correction
  E_dir(r) - E_long(r) over pairs closer than r_c, with E_dir the softened
  direct-sum field above.  Active ions inside the mesh take part.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module.
"""
from __future__ import annotations

import math
import tempfile
from pathlib import Path

import numpy as np
from scipy.spatial import cKDTree
from scipy.special import erf

COULOMB_CONST = 8.987551787e9     # utils/constants.h:20
EPSILON_0 = 8.854187817e-12       # utils/constants.h:19
DIRECT_SOFTENING_M = 1e-10        # SpaceChargeModelFactory.h:26


# ---------------------------------------------------------------------------
# direct summation
# ---------------------------------------------------------------------------
def direct_field(x, y, z, q, active, softening: float = DIRECT_SOFTENING_M, chunk: int = 512) -> np.ndarray:
    """[3, n] field of the direct summation (SpaceChargeDirectModel.cpp:20-66)."""
    n = x.shape[0]
    out = np.zeros((3, n))
    act = np.asarray(active) != 0
    idx = np.nonzero(act)[0]
    if n <= 1 or idx.size == 0:
        return out
    eps2 = softening * softening
    min_d2 = max(eps2 * 1e-4, 1e-30)
    px, py, pz, pq = x[idx], y[idx], z[idx], q[idx]
    for s in range(0, idx.size, chunk):
        ii = idx[s:s + chunk]
        dx = x[ii, None] - px[None, :]
        dy = y[ii, None] - py[None, :]
        dz = z[ii, None] - pz[None, :]
        r2 = dx * dx + dy * dy + dz * dz
        keep = (r2 >= min_d2) & (ii[:, None] != idx[None, :])
        r = np.sqrt(np.where(keep, r2, 1.0))
        scale = np.where(keep, COULOMB_CONST * pq[None, :] / (r2 + eps2) / r, 0.0)
        out[0, ii] = (dx * scale).sum(axis=1)
        out[1, ii] = (dy * scale).sum(axis=1)
        out[2, ii] = (dz * scale).sum(axis=1)
    return out


def direct_field_reference(x, y, z, q, active, softening: float = DIRECT_SOFTENING_M) -> np.ndarray:
    """The reference's own SpaceChargeDirectModel (compiled harness)."""
    from oracle import harness, write_state
    n = x.shape[0]
    st = {"x": x, "y": y, "z": z, "vx": np.zeros(n), "vy": np.zeros(n), "vz": np.zeros(n),
          "mass": np.full(n, 1e-25), "charge": q, "ccs": np.zeros(n), "active": np.asarray(active, dtype=np.float64),
          "t_death": np.full(n, -1.0), "t_arrival": np.full(n, -1.0)}
    with tempfile.TemporaryDirectory() as td:
        ip, op = Path(td) / "in.bin", Path(td) / "field.bin"
        write_state(ip, st)
        harness("direct", **{"in": ip, "out": op, "softening": repr(softening)})
        return np.fromfile(op, dtype=np.float64).reshape(3, n)


REF_P3M = Path(__file__).resolve().parent / "_ref" / "ref_p3m"


def periodic_pm_field_reference_gpu(x, y, z, q, lo, hi, n) -> np.ndarray:
    """The reference's own GPU solver (GPUSpaceChargeP3M, compiled from its
    sources into _ref/ref_p3m by oracle/Makefile): [3, N] field."""
    import subprocess
    m = x.shape[0]
    with tempfile.TemporaryDirectory() as td:
        ip, op = Path(td) / "ions.bin", Path(td) / "field.bin"
        with open(ip, "wb") as f:
            f.write(np.int64(m).tobytes())
            for a in (x, y, z, q):
                f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        args = [str(REF_P3M), f"in={ip}", f"out={op}", f"nx={n[0]}", f"ny={n[1]}", f"nz={n[2]}",
                f"xmin={lo[0]!r}", f"ymin={lo[1]!r}", f"zmin={lo[2]!r}",
                f"xmax={hi[0]!r}", f"ymax={hi[1]!r}", f"zmax={hi[2]!r}"]
        r = subprocess.run(args, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"ref_p3m failed ({r.returncode}): {r.stderr[-500:]}")
        return np.fromfile(op, dtype=np.float64).reshape(3, m)


# ---------------------------------------------------------------------------
# CIC helpers
# ---------------------------------------------------------------------------
def _cic(x, y, z, lo, inv_h, n):
    """Grid coordinates, base cell, float32 fractions, inside mask."""
    f = [(np.asarray(c) - lo[a]) * inv_h[a] for a, c in enumerate((x, y, z))]
    inside = np.ones(x.shape[0], dtype=bool)
    for a in range(3):
        inside &= (f[a] >= 0) & (f[a] < n[a] - 1)
    base = [np.where(inside, np.floor(np.where(inside, f[a], 0)).astype(np.int64), 0) for a in range(3)]
    return f, base, inside


def _corner_weights_f32(fr):
    """The eight CIC weights in float32, products taken left to right as
    (1-fx)*(1-fy)*(1-fz) etc. (GPUSpaceChargeP3M.cu:80-87)."""
    fx, fy, fz = (np.asarray(v, dtype=np.float32) for v in fr)
    one = np.float32(1.0)
    gx, gy, gz = one - fx, one - fy, one - fz
    w = {}
    for dx, ax in ((0, gx), (1, fx)):
        for dy, ay in ((0, gy), (1, fy)):
            for dz, az in ((0, gz), (1, fz)):
                w[(dx, dy, dz)] = (ax * ay * az).astype(np.float32)
    return w


def _corner_weights_f64(fr):
    fx, fy, fz = fr
    w = {}
    for dx, ax in ((0, 1.0 - fx), (1, fx)):
        for dy, ay in ((0, 1.0 - fy), (1, fy)):
            for dz, az in ((0, 1.0 - fz), (1, fz)):
                w[(dx, dy, dz)] = ax * ay * az
    return w


# ---------------------------------------------------------------------------
# the reference's periodic particle-mesh solver
# ---------------------------------------------------------------------------
def periodic_pm_field(x, y, z, q, lo, hi, n) -> np.ndarray:
    """[3, N] field of GPUSpaceChargeP3M::compute_space_charge_field_raw."""
    lo = np.asarray(lo, dtype=np.float64)
    ext = np.asarray(hi, dtype=np.float64) - lo
    nx, ny, nz = n
    inv_h = np.array([nx / ext[0], ny / ext[1], nz / ext[2]])
    h = ext / np.array(n)
    f, base, inside = _cic(x, y, z, lo, inv_h, n)
    i0, j0, k0 = base
    fr = [np.where(inside, f[a] - base[a], 0.0) for a in range(3)]
    w = _corner_weights_f32(fr)
    rho = np.zeros(n)
    for (dx, dy, dz), wc in w.items():
        np.add.at(rho, (i0[inside] + dx, j0[inside] + dy, k0[inside] + dz),
                  wc[inside].astype(np.float64) * q[inside])
    rho_hat = np.fft.rfftn(rho)
    nz_half = nz // 2 + 1
    lx, ly, lz = nx * h[0], ny * h[1], nz_half * 2 * h[2]
    ii = np.arange(nx)
    jj = np.arange(ny)
    kk = np.arange(nz_half)
    kx = np.where(ii < nx // 2, 2.0 * math.pi * ii / lx, 2.0 * math.pi * (ii - nx) / lx)
    ky = np.where(jj < ny // 2, 2.0 * math.pi * jj / ly, 2.0 * math.pi * (jj - ny) / ly)
    kz = 2.0 * math.pi * kk / lz
    k2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
    vol = h[0] * h[1] * h[2]
    scale = np.where(k2 < 1e-10, 0.0, 1.0 / (EPSILON_0 * np.where(k2 < 1e-10, 1.0, k2) * vol))
    phi = np.fft.irfftn(rho_hat * scale, s=n, axes=(0, 1, 2)) * (nx * ny * nz)   # unnormalised inverse, as cuFFT
    phi = phi * (1.0 / (nx * ny * nz))
    grids = []
    for a, d in enumerate(h):
        g = np.empty_like(phi)
        sl = [slice(None)] * 3

        def at(s):
            t = list(sl)
            t[a] = s
            return tuple(t)
        g[at(slice(1, -1))] = -(phi[at(slice(2, None))] - phi[at(slice(None, -2))]) / (2.0 * d)
        g[at(0)] = -(phi[at(1)] - phi[at(0)]) / d
        g[at(-1)] = -(phi[at(-1)] - phi[at(-2)]) / d
        grids.append(g)
    out = np.zeros((3, x.shape[0]))
    for c in range(3):
        acc = np.zeros(x.shape[0])
        for (dx, dy, dz), wc in w.items():
            vals = grids[c][np.where(inside, i0 + dx, 0), np.where(inside, j0 + dy, 0), np.where(inside, k0 + dz, 0)]
            acc += wc.astype(np.float64) * vals
        out[c] = np.where(inside, acc.astype(np.float32).astype(np.float64), 0.0)
    return out


# ---------------------------------------------------------------------------
# isolated P3M (this library's solver)
# ---------------------------------------------------------------------------
def e_long(r, alpha):
    """Long-range (mesh) part of the unit-charge field magnitude / COULOMB_CONST."""
    r = np.asarray(r, dtype=np.float64)
    safe = np.where(r > 0, r, 1.0)
    v = erf(alpha * safe) / (safe * safe) - (2.0 * alpha / math.sqrt(math.pi)) * np.exp(-(alpha * safe) ** 2) / safe
    return np.where(r > 0, v, 0.0)


def green_field(n, h, alpha) -> list[np.ndarray]:
    """Sampled long-range field of a unit charge at the origin on the
    zero-padded (2n)^3 grid, displacements wrapped to (-n, n); index n
    (never reached by data in [0, n)) is zero."""
    m = [2 * v for v in n]
    d = []
    for a in range(3):
        idx = np.arange(m[a])
        s = np.where(idx < n[a], idx, idx - m[a]).astype(np.float64)
        s[n[a]] = 0.0
        d.append(s * h[a])
    dx, dy, dz = np.meshgrid(d[0], d[1], d[2], indexing="ij")
    r = np.sqrt(dx * dx + dy * dy + dz * dz)
    f = COULOMB_CONST * e_long(r, alpha) / np.where(r > 0, r, 1.0)
    g = [f * dx, f * dy, f * dz]
    for a in range(3):
        for comp in g:
            sl = [slice(None)] * 3
            sl[a] = n[a]
            comp[tuple(sl)] = 0.0
    return g


def p3m_field(x, y, z, q, active, lo, h, n, alpha, rc, softening: float = DIRECT_SOFTENING_M) -> np.ndarray:
    """[3, N] isolated P3M field (mesh + particle-particle correction)."""
    lo = np.asarray(lo, dtype=np.float64)
    h = np.asarray(h, dtype=np.float64)
    n = tuple(int(v) for v in n)
    act = np.asarray(active) != 0
    f, base, inside = _cic(x, y, z, lo, 1.0 / h, n)
    use = inside & act
    i0, j0, k0 = base
    fr = [np.where(use, f[a] - base[a], 0.0) for a in range(3)]
    w = _corner_weights_f64(fr)
    m = tuple(2 * v for v in n)
    rho = np.zeros(m)
    for (dx, dy, dz), wc in w.items():
        np.add.at(rho, (i0[use] + dx, j0[use] + dy, k0[use] + dz), wc[use] * q[use])
    rho_hat = np.fft.rfftn(rho)
    out = np.zeros((3, x.shape[0]))
    for c, g in enumerate(green_field(n, h, alpha)):
        e = np.fft.irfftn(rho_hat * np.fft.rfftn(g), s=m, axes=(0, 1, 2))
        acc = np.zeros(x.shape[0])
        for (dx, dy, dz), wc in w.items():
            acc += wc * e[np.where(use, i0 + dx, 0), np.where(use, j0 + dy, 0), np.where(use, k0 + dz, 0)]
        out[c] = np.where(use, acc, 0.0)
    # particle-particle correction
    ids = np.nonzero(use)[0]
    if ids.size > 1:
        pts = np.stack([x[ids], y[ids], z[ids]], axis=1)
        pairs = cKDTree(pts).query_pairs(rc, output_type="ndarray")
        if pairs.size:
            a, b = ids[pairs[:, 0]], ids[pairs[:, 1]]
            d = np.stack([x[a] - x[b], y[a] - y[b], z[a] - z[b]])
            r2 = (d * d).sum(axis=0)
            eps2 = softening * softening
            ok = (r2 >= max(eps2 * 1e-4, 1e-30)) & (r2 < rc * rc)
            r = np.sqrt(np.where(ok, r2, 1.0))
            s = np.where(ok, COULOMB_CONST * (1.0 / (r2 + eps2) - e_long(r, alpha)) / r, 0.0)
            for c in range(3):
                np.add.at(out[c], a, d[c] * s * q[b])
                np.add.at(out[c], b, -d[c] * s * q[a])
    return out
