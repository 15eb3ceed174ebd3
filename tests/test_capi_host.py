"""CPU-side checks of the product library: it loads, exports every symbol
include/icarion_b200.h declares, the ctypes layer matches the header, and
the host logic (config loading, sharding) behaves as specified.  No kernel
is launched here."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from icarion_b200 import _capi as capi
from icarion_b200 import config as cfg
from icarion_b200 import parallel

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "icarion_b200.h"


def declared_functions() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(icb_[a-z0-9_]+)\s*\(", text))


def test_library_loads_and_exports_every_declared_symbol():
    lib = capi.lib()
    names = declared_functions()
    assert names, "no declarations parsed"
    out = subprocess.run(["nm", "-D", "--defined-only", str(capi.LIB_PATH)], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (icb_[a-z0-9_]+)", out))
    missing = names - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    for n in names:
        assert hasattr(lib, n)


def test_ctypes_signatures_cover_header():
    assert declared_functions() == set(capi.SIGNATURES), (
        declared_functions() ^ set(capi.SIGNATURES))


def test_struct_sizes_match_c_layout():
    # compile a tiny C program against the header and compare sizeof
    src = r'''
    #include "icarion_b200.h"
    #include <stdio.h>
    #include <stddef.h>
    int main(void){printf("%zu %zu %zu %zu %zu %zu\n", sizeof(icb_ensemble_params), sizeof(icb_config),
        sizeof(icb_run_stats), sizeof(icb_species_spec), sizeof(icb_ipm_config),
        offsetof(icb_ipm_config, net_E_min_J)); return 0;}'''
    tmp = Path(subprocess.run(["mktemp", "-d"], capture_output=True, text=True).stdout.strip())
    (tmp / "s.c").write_text(src)
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(tmp / "s.c"), "-o", str(tmp / "s")], check=True)
    sizes = [int(v) for v in subprocess.run([str(tmp / "s")], capture_output=True, text=True).stdout.split()]
    assert sizes == [C.sizeof(capi.EnsembleParams), C.sizeof(capi.Config), C.sizeof(capi.RunStats),
                     C.sizeof(capi.SpeciesSpec), C.sizeof(capi.IpmConfig), capi.IpmConfig.net_E_min_J.offset]


def test_abi_version_and_error_reporting_without_compute():
    lib = capi.lib()
    assert lib.icb_abi_version() == 10
    # invalid configuration is rejected before any device work
    h = C.c_void_p()
    c = capi.Config()
    c.n_ensembles = 0
    rc = lib.icb_create(C.byref(c), C.byref(h))
    assert rc == capi.ICB_ERR_INVALID_ARGUMENT
    assert b"n_ensembles" in lib.icb_last_error()
    with pytest.raises(capi.IcbError):
        capi.check(rc)


def test_config_loader_reads_reference_schema(tmp_path):
    raw = {
        "simulation": {"total_time_s": 5e-5, "dt_s": 5e-10, "write_interval": 1000, "integrator": "Boris",
                       "enable_gpu": True, "rng_seed": 123},
        "physics": {"collision_model": "HSS", "enable_space_charge": False},
        "ions": {"species": [{"id": "X200", "count": 4096,
                              "position": {"type": "gaussian", "center": [0, 0, 0], "std": [5e-4] * 3},
                              "velocity": {"type": "thermal", "temperature_K": 300.0}}]},
        "domains": [{"name": "drift", "instrument": "IMS",
                     "geometry": {"origin_m": [0, 0, -0.01], "length_m": 0.1, "radius_m": 0.05},
                     "env": {"temperature_K": 300.0, "pressure_Pa": 1000.0, "gas_species": "N2"},
                     "fields": {"DC": {"EN_Td": 20.0}}}],
    }
    db = {"species": {"X200": {"mass_amu": 200.0, "charge": 1, "CCS_A2": 150.0}}}
    rc = cfg.load(raw, species_db=db)
    assert rc.n_steps == 100000 and rc.enable_gpu and rc.collision_model == capi.COLLISION_HSS
    sp, count, pos, vel = rc.species[0]
    assert count == 4096 and sp.mass_kg == 200.0 * cfg.AMU_TO_KG and sp.ccs_m2 == 150.0 * cfg.ANGSTROM2_TO_M2
    e = cfg.ensemble_params(rc.domain, sp.sigma_for_gas("N2"), rc.dt_s)
    assert abs(e["axial_V"] / e["length_m"] - 4828.6470106932802) < 1e-9
    st = cfg.to_struct(e)
    assert st.instrument == capi.INSTRUMENT_IMS and st.dt_s == 5e-10


def test_shard_ranges_cover_all_ions():
    for n in (1, 7, 4096, 1_000_003):
        for w in (1, 2, 3, 8):
            spans = [parallel.shard_range(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(w - 1))
            assert max(e - b for b, e in spans) - min(e - b for b, e in spans) <= 1
    off = np.array([0, 10, 25, 40], dtype=np.uint64)
    assert parallel.shard_offsets(off, 12, 30).tolist() == [0, 0, 13, 18]


def test_collision_substeps_need_the_plain_form():
    """Collision sub-steps run in the plain per-step form only; the
    null-collision forms reject them before any device work, and so does a
    count outside [0, 1024]."""
    import sys
    sys.path.insert(0, str(ROOT / "tests"))
    from helpers import config0_ensemble
    ens = (capi.EnsembleParams * 1)(cfg.to_struct(config0_ensemble()))
    for coll, sub, rc in ((capi.COLLISION_HSS, 4, capi.ICB_ERR_UNSUPPORTED),
                          (capi.COLLISION_HSS_PLAIN, 2000, capi.ICB_ERR_INVALID_ARGUMENT),
                          (capi.COLLISION_HSS_PLAIN, -1, capi.ICB_ERR_INVALID_ARGUMENT)):
        c = capi.Config()
        c.precision = capi.PREC_FP64
        c.integrator = capi.INTEGRATOR_BORIS
        c.collision_model = coll
        c.n_ensembles = 1
        c.ensembles = C.cast(ens, C.POINTER(capi.EnsembleParams))
        c.collision_subcycles = sub
        h = C.c_void_p()
        assert capi.lib().icb_create(C.byref(c), C.byref(h)) == rc
        assert "collision" in capi.lib().icb_last_error().decode()


def test_per_ion_philox_rounds_equal_the_generator():
    """The kernel forms the candidate draws' first two Philox rounds once per
    ion (icb_rng.cuh: philox_ion_setup / philox_ion); on random keys, ions,
    steps and both candidate substreams the words equal Philox4x32-10's
    (compiled on the host from the same header), and those equal the
    oracle's generator."""
    import sys
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    src = r'''
    #include <cstdio>
    #include <cstdint>
    #include "icb_rng.cuh"
    using namespace icb;
    int main() {
        uint64_t x = 0x9E3779B97F4A7C15ull;
        auto next = [&]() { x ^= x << 13; x ^= x >> 7; x ^= x << 17; return x; };
        for (int t = 0; t < 4000; ++t) {
            const uint64_t seed = next();
            uint32_t rk[20];
            philox_round_keys(seed, rk);
            const uint32_t id = static_cast<uint32_t>(next()), step = static_cast<uint32_t>(next());
            const PhiloxIon q = philox_ion_setup(id, rk);
            for (uint32_t s = 0; s < 2; ++s) {
                const U4 a = philox4x32_10_rk(id, step, s, 0u, rk), b = philox_ion(q, step, s, rk);
                if (a.x != b.x || a.y != b.y || a.z != b.z || a.w != b.w) return 1;
                if (t < 16) std::printf("%llu %u %u %u %u %u %u %u\n", (unsigned long long)seed, id, step, s,
                                        a.x, a.y, a.z, a.w);
            }
        }
        return 0;
    }'''
    tmp = Path(subprocess.run(["mktemp", "-d"], capture_output=True, text=True).stdout.strip())
    (tmp / "p.cpp").write_text(src)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(ROOT / "icarion_b200" / "csrc"), str(tmp / "p.cpp"),
                    "-o", str(tmp / "p")], check=True)
    out = subprocess.run([str(tmp / "p")], capture_output=True, text=True)
    assert out.returncode == 0, "per-ion rounds differ from Philox4x32-10"
    lines = out.stdout.splitlines()
    assert len(lines) == 32
    for line in lines:
        seed, idv, step, s, *words = (int(v) for v in line.split())
        ctr = np.array([[idv, step, s, 0]], dtype=np.uint32)
        assert np.array_equal(orc.philox(ctr, seed)[0], np.array(words, dtype=np.uint32))
