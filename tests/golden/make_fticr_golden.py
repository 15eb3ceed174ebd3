"""Generate tests/golden/fticr_sc_direct.npz: the reference's own Boris push
in the FT-ICR cell with and without its direct space charge.

    make -C oracle REF=<reference tree> && python tests/golden/make_fticr_golden.py

What runs: ``oracle/_ref/ref_harness run`` — BorisStrategy, the FTICR field
model (AnalyticalFieldModel.cpp:174-186) and the uniform 7 T field, with
``sc=direct``: SpaceChargeDirectModel (SpaceChargeDirectModel.cpp:20-66,
softening 1e-10 m) updated once per step and added as q E_sc by the force
registry; collisions off (the cell's 1e-7 Pa He gives ~1e-5 collisions per
ion over the run).

Cell: the FT-ICR workload (icarion_b200.fticr.fticr_cell) with 1,024 ions,
m/z uniform over 500-1500, a 0.5 mm Gaussian cloud 2 mm off axis on its
cyclotron orbit; dt = 1e-9 s, 20,000 steps.  The space-charge displacement
of each ion is the difference of the two final states.
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))
import oracle as orc  # noqa: E402
from make_golden import save  # noqa: E402

from icarion_b200 import fticr  # noqa: E402

N_IONS, STEPS, DT, SIGMA = 1024, 20000, 1e-9, 5e-4
DOMAIN = dict(instrument="FTICR", origin_z=0.0, length=0.05, radius=0.025, T=300, P=1e-7, gas="He",
              radial_V=1.0, magnetic=1, B_z=7.0)


def main() -> None:
    if not orc.have_harness():
        raise SystemExit("oracle/_ref/ref_harness missing: run `make -C oracle REF=<reference tree>`")
    cell = fticr.fticr_cell(n_ions=N_IONS, cloud_sigma_m=SIGMA)
    st = cell.ions
    s0 = {k: np.array(getattr(st, k), dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "charge")}
    s0["ccs"] = np.full(st.n, 1e-20)
    s0["active"] = np.ones(st.n)
    out = {}
    for sc in ("none", "direct"):
        t0 = time.time()
        fin, stats, _ = orc.harness_run(s0, STEPS, DOMAIN, integrator="boris", collision="none", dt=DT, sc=sc)
        print(f"reference FT-ICR run sc={sc}: {time.time() - t0:.1f} s", flush=True)
        out[sc] = fin
    save("fticr_sc_direct.npz", **{f"in_{k}": s0[k] for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "charge")},
         **{f"nosc_{k}": out["none"][k] for k in ("x", "y", "z", "vx", "vy", "vz", "active")},
         **{f"sc_{k}": out["direct"][k] for k in ("x", "y", "z", "vx", "vy", "vz", "active")},
         steps=STEPS, dt=DT, n_ions=N_IONS, sigma_m=SIGMA, softening_m=1e-10)


if __name__ == "__main__":
    main()
