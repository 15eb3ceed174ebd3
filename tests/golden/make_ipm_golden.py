"""Generate tests/golden/ipm_ref_40Td.npz: the reference's own interaction-
potential collision handler run on the config-3 potential.

    make -C oracle REF=<reference tree> && python tests/golden/make_ipm_golden.py [--quick]

What runs: ``oracle/_ref/ref_harness`` with ``collision=ipm`` — the
reference's InteractionPotentialCollisionHandler (compiled unchanged from
src/core/physics/collisions/InteractionPotentialCollisionHandler.cpp) driven
by the reference engine's per-step order, Boris push, random orientation
mode.  Its offline sample set is built here by the reference tool's per-cell
rule (tools/interaction_potential_precompute.cpp:2692-2880): one orientation
(the potential is isotropic), relative speeds on a log grid, impact points
uniform over a disk of radius b_max = 12 A (the event cross-section
pi b_max^2 of every cell), momentum transfers dp = mu (v_out - v0) with the
deflection from the restated quadrature (oracle/icb_oracle.c
orc_ipm_chi_quad), equal-weight CDFs.  The impact points are stratified
(one per equal-area annulus, 16,384 per cell): the tool's independent draws
leave Monte Carlo errors of 1-7 % in each cell's momentum-transfer cross
section (0.5 % in the drift at 4,096 draws per cell), stratification the
same uniform-area law without them.  The file is read by the project's
definition of the reference's loader (oracle/ref_ipm_loader.cpp); it is a
temporary and not kept.

Physics (config 3 potential; the ion of the learned-IPM evaluation):
300 Da, +1 ions in N2 at 300 K and 1000 Pa, E/N = 40 Td, LJ 12-6 (5 meV at
4 A) + C4 of the N2 polarisability 1.74 A^3; dt = 1e-10 s (collision
probability per step ~6 %); 65,536 ions (seed-123 IonLoader cloud, sigma
0.5 mm, thermal velocities) x 30,000 steps; moments every 1,000 steps,
displacement reference after 6,000 steps.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))
import oracle as orc  # noqa: E402
from make_golden import AMU, init_state, save  # noqa: E402

from icarion_b200 import ipm  # noqa: E402

KB = 1.380649e-23
EN_TD = 40.0
DOMAIN = dict(instrument="IMS", origin_z=-0.01, length=0.1, radius=0.05, T=300, P=1000, gas="N2", EN_Td=EN_TD)
ION_MASS_DA = 300.0
GAS_MASS_DA = 28.0134
DT = 1e-10
SEED = 123
# sample set: relative speeds 0.05 .. 6 x the mean thermal relative speed
# sqrt(8 kT / (pi mu)) (the tool's default grid is 0.2 .. 5 x, 32 bins)
G_LO, G_HI, N_BINS, N_TRIALS, SET_SEED = 0.05, 6.0, 96, 16384, 7


def sample_set_params() -> dict:
    s = ipm.IpmSetup()
    c12, c6, c4 = s.coefficients()
    mi, mn = ION_MASS_DA * AMU, GAS_MASS_DA * AMU
    mu = mi * (mn / (mi + mn))
    vth = math.sqrt(8.0 * KB * 300.0 / (math.pi * mu))
    return dict(c12=c12, c6=c6, c4=c4, sigma=s.r_m_m * 2.0 ** (-1.0 / 6.0), mu=mu, g_min=G_LO * vth,
                g_max=G_HI * vth, n_bins=N_BINS, b_max=s.b_max_m, n_trials=N_TRIALS, seed=SET_SEED, stratified=True)


def main(quick: bool) -> None:
    if not orc.have_harness():
        raise SystemExit("oracle/_ref/ref_harness missing: run `make -C oracle REF=<reference tree>`")
    n, steps = (8192, 10000) if quick else (65536, 30000)
    snap, ref_step = 1000, steps // 5
    p = sample_set_params()
    with tempfile.TemporaryDirectory() as td:
        path = Path(td) / "ipm_samples.bin"
        info = orc.write_ipm_sample_set(path, **p)
        s0 = init_state(n, seed=SEED, mass_amu=ION_MASS_DA)
        t0 = time.time()
        fin, stats, mom = orc.harness_run(s0, steps, DOMAIN, integrator="boris", collision="ipm",
                                          ipm_samples=str(path), dt=DT, seed=SEED, snap=snap, ref_step=ref_step,
                                          threads=8)
        print(f"reference IPM run: {time.time() - t0:.1f} s, {stats}", flush=True)
    save("ipm_ref_40Td.npz", moments=mom, snap_every=snap, ref_step=ref_step, steps=steps, dt=DT, n_ions=n,
         seed=SEED, ion_mass_amu=ION_MASS_DA, collisions=stats["collisions"], ion_steps_per_s=stats["ion_steps_per_s"],
         threads=stats["threads"], domain=json.dumps(DOMAIN), final_active=fin["active"],
         sample_set=json.dumps({k: v for k, v in p.items()}), logv_bins=info["logv_bins"],
         sigma_mt_m2=info["sigma_mt_m2"])


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    main(ap.parse_args().quick)
