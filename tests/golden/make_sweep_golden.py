"""Generate tests/golden/sweep_ref.npz: the reference's own Boris + HSS code
on one ensemble of each species of the batched E/N sweep.

    make -C oracle REF=<reference tree> && python tests/golden/make_sweep_golden.py [--quick]

What runs: ``oracle/_ref/ref_harness run`` (BorisStrategy,
HSSCollisionHandler with PhysicsRng(seed + ion index), the IMS field model,
the engine's per-step order) for ensembles 30, 31 and 32 of the default
sweep (icarion_b200.sweep.en_sweep): 12.9, 13.7 and 14.6 Td with the
species (100 Da, 100 A^2), (500 Da, 250 A^2) and (2000 Da, 600 A^2), N2 at
300 K and 1000 Pa, each with the sweep's own dt = 0.1 / nu_max.  4,096 ions
per ensemble (the seed-123 IonLoader cloud of that species: 0.5 mm, thermal),
50,000 steps, moments every 1,000 steps, displacement reference after 10,000.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))
import oracle as orc  # noqa: E402
from make_golden import AMU, save  # noqa: E402

from icarion_b200 import sweep  # noqa: E402

ENSEMBLES = (30, 31, 32)


def main(quick: bool) -> None:
    if not orc.have_harness():
        raise SystemExit("oracle/_ref/ref_harness missing: run `make -C oracle REF=<reference tree>`")
    n, steps = (1024, 10000) if quick else (4096, 50000)
    snap, ref_step = 1000, steps // 5
    sw = sweep.en_sweep(n_ensembles=64, counts=np.full(64, 16))
    out = {}
    for e in ENSEMBLES:
        m_da, ccs_a2 = sweep.SPECIES[int(sw.species[e])]
        en = float(sw.en_td[e])
        dt = float(sw.ensembles[e]["dt_s"])
        dom = dict(instrument="IMS", origin_z=-0.01, length=0.1, radius=0.05, T=300, P=1000, gas="N2", EN_Td=en)
        p = Path(__file__).resolve().parent / "_tmp_sweep_init.bin"
        orc.harness("init", seed=123, n=n, sigma_pos=5e-4, T=300, mass=repr(m_da * AMU), ccs=repr(ccs_a2 * 1e-20),
                    out=p)
        s0 = orc.read_state(p)
        p.unlink()
        t0 = time.time()
        fin, stats, mom = orc.harness_run(s0, steps, dom, integrator="boris", collision="hss", dt=repr(dt), seed=123,
                                          snap=snap, ref_step=ref_step, zdet=2.0e-3, threads=8)
        print(f"ensemble {e}: {time.time() - t0:.1f} s, {stats}", flush=True)
        out[e] = dict(moments=mom, collisions=stats["collisions"], en_td=en, dt=dt, mass_amu=m_da, ccs_a2=ccs_a2,
                      domain=json.dumps(dom))
    arrays = {}
    for e, d in out.items():
        for k, v in d.items():
            arrays[f"e{e}_{k}"] = v
    save("sweep_ref.npz", ensembles=np.array(ENSEMBLES), n_ions=n, steps=steps, snap_every=snap, ref_step=ref_step,
         seed=123, **arrays)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    main(ap.parse_args().quick)
