"""Benchmark of the B200 batch step on the mixed-precision IMS workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU): 1,048,576 ions of 200 Da, +1, HSS cross-section 150 A^2,
in N2 at 300 K and 1000 Pa, uniform E at 20 Td, Boris push, dt = 5e-10 s,
collisions by the null-collision HSS scheme with Philox; velocities, field
and collision arithmetic in FP32, positions and time in FP64.  One bench
step = 1,000 engine steps of all ions (the engine's snapshot interval), so
the default 100 timed steps are the workload's full 100,000-step run.
Inputs are synthetic (the reference's own ion loader semantics, seed 123).

Metric: ion-steps/s (whole job).  Timed on the device with CUDA events on
the launching stream, L2 flushed (256 MB write) between timed steps, barrier
+ synchronize around the timed loop, max over ranks.  Under torchrun each
rank advances its own 1,048,576 ions (weak scaling; ion ids offset by rank)
and the per-snapshot ensemble moments are all-reduced over NCCL.

--impl reference runs the reference's own CPU code (oracle/_ref/ref_harness,
compiled from the reference sources) on all host cores for the same metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
N_IONS = 1_048_576
STEPS_PER_BENCH_STEP = 1000
DT = 5e-10
EN_TD = 20.0
METRIC = "ion-steps/s on 1 B200: mixed-prec vs plain FP64 at <=0.3% K0 error"
SWEEP_WORKLOAD = ("E/N sweep, 64 ensembles (2-100 Td log-spaced, N2 300 K 1000 Pa), species 100/500/2000 Da "
                  "(100/250/600 A^2) round-robin, {n:,} ions (log-uniform 1k-256k per ensemble, seed 123), "
                  "dt = 0.1/nu_max per ensemble, Boris + HSS")
WORKLOAD = "IMS drift, 1,048,576 ions (200 Da, +1, 150 A^2 HSS) in N2 300 K 1000 Pa, 20 Td, Boris + HSS, dt 5e-10 s"
# trapped IMS on the time-dependent field path (TIMSAxialFieldModel): 20 mm
# tube, axial profile 0 -> -4495 V/m ramped to zero over 10..40 us, RF
# 180 V at 2 MHz (r0 5 mm), axial gas flow 134 m/s, N2 300 K 310 Pa
TIMS_DOMAIN = {"instrument": "TIMS", "geometry": {"origin_m": [0.0, 0.0, -0.01], "length_m": 0.02, "radius_m": 0.005},
               "env": {"temperature_K": 300.0, "pressure_Pa": 310.0, "gas_species": "N2",
                       "flow_model": "axial_uniform", "axial_flow_velocity_m_s": 134.0},
               "fields": {"RF": {"voltage_V": 180.0, "frequency_Hz": 2.0e6}, "DC": {"quad_V": 0.0},
                          "TIMS": {"z_positions_m": [0.0, 0.02], "axial_field_initial_profile_V_m": [0.0, -4495.0],
                                   "axial_field_final_profile_V_m": [0.0, 0.0], "ramp_start_s": 1.0e-5,
                                   "ramp_end_s": 4.0e-5, "ramp_mode": "linear"}}}
TIMS_WORKLOAD = ("TIMS ramp, 1,048,576 ions (200 Da, +1, 150 A^2 HSS) in N2 300 K 310 Pa against 134 m/s flow, "
                 "profile 0..-4495 V/m ramped over 10-40 us, RF 180 V 2 MHz, Boris + HSS, dt 5e-10 s")
# Algorithmic bytes each ion moves per launch of the fused kernel:
# read  x,y,z(24) v(12) tau,Q*(8) next,start(8) mass,charge(16) flags(1) t_arr(8) = 77
# write x,y,z(24) v(12) tau,Q*(8) next,start(8) flags(1)                          = 53
# (hi/lo: positions 6 floats = 24 B as well; FP64: v and the clock are doubles: 97 + 73)
BYTES_PER_ION_LAUNCH = {"mixed": 130, "hilo": 130, "fp64": 170}
STEPPING = {"events": 0, "per-step": 1, "events-all": 2}
# ncu summary of the fused mixed launch (1,048,576 ions x 1000 steps, event
# form).  Its "bench figures" block holds the warp instructions
# (smsp__inst_executed.sum) and DRAM bytes (dram__bytes_read.sum +
# dram__bytes_write.sum) of one launch, and the kernel_source_hash of the
# sources the capture ran; the figures are used only while that hash matches
# the current sources.
PROFILE_FUSED = "profiles/k_step_mixed_fused_ims_1M.md"
PROFILE_STEP1 = "profiles/k_step1_ws_mixed_per_step_16M.md"


def profile_figures(rel: str, unit: str = "icb_step_mixed.cu") -> dict:
    """Figures of a committed ncu summary and whether they belong to the
    kernel as built now."""
    import re
    sys.path.insert(0, str(ROOT))
    from icarion_b200.build import kernel_source_hash
    path = ROOT / rel
    txt = path.read_text() if path.exists() else ""
    m = re.search(r"<!-- bench figures\n(.*?)-->", txt, re.S)
    figs = {}
    for line in (m.group(1).splitlines() if m else []):
        if ":" in line:
            k, v = line.split(":", 1)
            figs[k.strip()] = v.strip()
    fresh = bool(figs) and figs.get("source_sha256") == kernel_source_hash(unit)
    out = {"file": rel, "fresh": fresh}
    if fresh:
        for key in ("inst_per_launch", "dram_bytes_per_launch"):
            if key in figs:
                out[key] = float(figs[key])
    else:
        out["note"] = ("no figures block" if not figs else
                       "stale: the summary was taken of other kernel sources; its figures are not used")
    return out


def issue_roofline(args, avg_launch_ms: float, clk: dict, prof: dict) -> dict | None:
    """Instruction-issue roofline of the fused mixed kernel: warp
    instructions per launch (ncu summary of the same workload, current
    sources only) / live launch time, against 4 schedulers x SMs x the SM
    clock sampled during the run."""
    if args.precision != "mixed" or args.steps_per_launch != 1000 or args.workload != "ims-1M" \
            or args.stepping != "events" or not prof.get("fresh"):
        return None
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    inst = prof["inst_per_launch"]
    achieved = inst / (avg_launch_ms * 1e-3)
    peak = 4.0 * sms * mhz * 1e6
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "warp instructions/s",
            "frac": achieved / peak, "inst_per_launch": inst, "sms": sms, "sm_mhz": mhz,
            "source": f"smsp__inst_executed.sum of one launch ({prof['file']}); peak = 4 x SMs x sampled SM clock"}


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                      "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                     stderr=subprocess.DEVNULL, text=True)
        self.thr = threading.Thread(target=self._read, daemon=True)
        self.thr.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# reference CPU code (oracle/_ref/ref_harness)
# ---------------------------------------------------------------------------
REF_DOMAIN = dict(instrument="IMS", origin_z=-0.01, length=0.1, radius=0.05, T=300, P=1000, gas="N2", EN_Td=EN_TD)


def _harness():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc  # noqa: E402  (CPU-baseline leg only)
    return orc


def reference_sample(n_ions: int, n_steps: int, threads: int, schedule: str = "static") -> dict:
    """Run the reference's Boris + HSS code on n_ions for n_steps; returns the
    harness's own loop timing.  schedule "static": the best CPU form (one
    OpenMP loop per step, push then collide per ion); "faithful": the engine's
    order as written (serial Boris loop, SimulationEngineIntegration.cpp:
    114-146, then the OpenMP collision loop, SimulationEngineCollisionRuntime
    .cpp:103-105)."""
    orc = _harness()
    with tempfile.TemporaryDirectory() as td:
        sp = Path(td) / "s.bin"
        orc.harness("init", seed=123, n=n_ions, sigma_pos=5e-4, T=300, mass=repr(200.0 * 1.66053906660e-27), out=sp)
        out = orc.harness("run", **{"in": sp, "out": Path(td) / "o.bin"}, **REF_DOMAIN, integrator="boris",
                          collision="hss", dt=DT, steps=n_steps, threads=threads, seed=123, schedule=schedule)
    return json.loads(out.strip().splitlines()[-1])


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(budget_s: float = 12.0) -> dict:
    """Bounded samples of the same workload on the host cores (rank 0, N=1):
    the reference code in its best CPU form (the reported value) and in the
    engine's own order."""
    orc = _harness()
    threads = cpu_threads()
    n = 65536
    if not orc.have_harness():
        return {"value": None, "unit": "ion-steps/s", "cores": threads, "kind": "reference",
                "sample": "unavailable: oracle/_ref/ref_harness was not built"}
    out = {}
    for schedule in ("static", "faithful"):
        probe = reference_sample(n, 20, threads, schedule)
        rate = max(probe["ion_steps_per_s"], 1.0)
        steps = int(min(max(budget_s * rate / n, 20), 100000))
        out[schedule] = (reference_sample(n, steps, threads, schedule), steps)
    (r, steps), (rf, steps_f) = out["static"], out["faithful"]
    return {"value": r["ion_steps_per_s"], "unit": "ion-steps/s", "cores": threads, "kind": "reference",
            "cpu_model": cpu_model(),
            "sample": f"{n} ions x {steps} steps of the same physics (reference BorisStrategy + HSSCollisionHandler, "
                      f"best CPU form: one OpenMP loop over ions per step, {threads} threads, {r['wall_s']:.1f} s)",
            "faithful_engine_order": {"value": rf["ion_steps_per_s"], "unit": "ion-steps/s",
                                      "sample": f"{n} ions x {steps_f} steps, serial Boris loop then the OpenMP "
                                                f"collision loop (the engine's order), {threads} threads, "
                                                f"{rf['wall_s']:.1f} s"}}


def run_reference_arm(args) -> None:
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    orc = _harness()
    threads = cpu_threads()
    line = {"impl": "reference", "metric": METRIC, "unit": "ion-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic"}
    if not orc.have_harness():
        line["unavailable"] = "reference CPU code was not compiled (oracle/_ref/ref_harness missing)"
        print(json.dumps(line))
        return
    n = 65536
    probe = reference_sample(n, 10, threads)
    rate = max(probe["ion_steps_per_s"], 1.0)
    per_step_s = min(1.0, 150.0 / max(args.steps + args.warmup, 1))
    sub = int(max(5, per_step_s * rate / n))
    for _ in range(args.warmup):
        reference_sample(n, sub, threads)
    wall, ion_steps = 0.0, 0
    for _ in range(args.steps):
        r = reference_sample(n, sub, threads)
        wall += r["wall_s"]
        ion_steps += r["ion_steps"]
    value = ion_steps / wall
    line.update({"value": value, "ms_per_step": 1e3 * wall / args.steps,
                 "config": {"workload": WORKLOAD, "ions": n, "engine_steps_per_bench_step": sub,
                            "sample": f"{n} of {N_IONS} ions per step (bounded CPU sample)"},
                 "cpu_baseline": {"value": value, "unit": "ion-steps/s", "cores": threads, "kind": "reference",
                                  "cpu_model": cpu_model(),
                                  "sample": f"{n} ions x {sub} engine steps per bench step (best CPU form: one "
                                            f"OpenMP loop over ions per step)"},
                 "e2e": {"value": value, "unit": "ion-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args) -> None:
    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from icarion_b200 import _capi as capi
    from icarion_b200 import config as cfg
    from icarion_b200 import parallel
    from icarion_b200.sim import IonState, Simulation, generate_ions

    rank, world, local = _env_rank()
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    prec_id = {"mixed": capi.PREC_MIXED, "fp64": capi.PREC_FP64, "hilo": capi.PREC_MIXED_HILO}[args.precision]

    tf_domain = None
    if args.workload == "en-sweep":
        # batched E/N sweep: 64 ensembles in one launch sequence (CUDA graphs, autotuned shape)
        from icarion_b200 import sweep
        sw = sweep.en_sweep()
        ensembles, st0, offsets, n_ions = sw.ensembles, sw.ions, sw.offsets, sw.n_ions
        workload = SWEEP_WORKLOAD.format(n=n_ions)
        args.graphs, args.autotune = True, True
    elif args.workload == "tims-1M":
        # trapped IMS: axial profile ramped over 10..40 us against a 134 m/s
        # axial gas flow, RF radial confinement (the time-dependent field path)
        tf_domain = TIMS_DOMAIN
        ensembles = [cfg.ensemble_params(tf_domain, 150e-20, DT, detector_z_m=1e30)]
        spec = cfg.species_spec(N_IONS, 200.0 * cfg.AMU_TO_KG, cfg.ELEM_CHARGE_C,
                                {"type": "gaussian", "center": [0, 0, 0], "std": [5e-4] * 3},
                                {"type": "thermal", "temperature_K": 300.0})
        st0, offsets, n_ions, workload = generate_ions(123, [spec]), None, N_IONS, TIMS_WORKLOAD
    else:
        domain = {"instrument": "IMS", "geometry": {"origin_m": [0.0, 0.0, -0.01], "length_m": 0.1, "radius_m": 0.05},
                  "env": {"temperature_K": 300.0, "pressure_Pa": 1000.0, "gas_species": "N2"},
                  "fields": {"DC": {"EN_Td": EN_TD}}}
        ensembles = [cfg.ensemble_params(domain, 150e-20, DT, detector_z_m=2.0e-3)]
        spec = cfg.species_spec(N_IONS, 200.0 * cfg.AMU_TO_KG, cfg.ELEM_CHARGE_C,
                                {"type": "gaussian", "center": [0, 0, 0], "std": [5e-4] * 3},
                                {"type": "thermal", "temperature_K": 300.0})
        st0, offsets, n_ions, workload = generate_ions(123, [spec]), None, N_IONS, WORKLOAD
    first_id = rank * n_ions
    n_ens = len(ensembles)
    # a dedicated (non-default) stream: the library launches on it, and the
    # timing events and the L2 flush are recorded on it too
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def make_sim(prec, K=args.steps_per_launch, collision=capi.COLLISION_HSS, stepping=None):
        s = Simulation(ensembles, precision=prec, integrator=capi.INTEGRATOR_BORIS, collision=collision,
                       rng_seed=123, device=dev, steps_per_launch=K, block_size=args.block,
                       pending_threshold=args.pending, steps_per_vote=args.spv, use_graphs=int(args.graphs),
                       stepping=STEPPING[args.stepping] if stepping is None else stepping)
        s.set_stream(stream.cuda_stream)
        if tf_domain is not None:
            s.apply_time_fields(0, tf_domain)
        s.upload(st0, ens_offsets=offsets, first_id=first_id)
        return s

    def timed_loop(sim, n_steps, steps_per_bench, allreduce=True):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n_steps)]
        kernel_ms, launches, timed_launches = 0.0, 0, 0
        stats_tot = {"candidates": 0, "collisions": 0}
        for i in range(n_steps):
            flush.zero_()
            ev[i][0].record(stream)
            rs = sim.advance(steps_per_bench)
            ev[i][1].record(stream)
            if allreduce and world > 1:
                parallel.allreduce_moments(sim.moments())
            kernel_ms += rs["step_kernel_ms"]
            launches += rs["kernel_launches"]
            timed_launches += min(math.ceil(steps_per_bench / sim_K(sim)), 64)
            for k in stats_tot:
                stats_tot[k] += rs[k]
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        return ms, kernel_ms, launches, timed_launches, stats_tot

    def sim_K(sim):
        return args.steps_per_launch if args.steps_per_launch > 0 else 1000

    sim = make_sim(prec_id)
    tuning = sim.autotune(500) if args.autotune else None
    # warm-up (same workload), then restart from the initial state
    for _ in range(args.warmup):
        sim.advance(STEPS_PER_BENCH_STEP)
    sim.upload(st0, ens_offsets=offsets, first_id=first_id)
    sim.set_clock(0, np.zeros(n_ens))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(dev)).split(",")[0]) if world == 1 else dev)
    clocks.start()
    ms, kernel_ms, launches, timed_launches, stt = timed_loop(sim, args.steps, STEPS_PER_BENCH_STEP)
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    ms_max = parallel.max_over_ranks(ms)
    ion_steps = n_ions * STEPS_PER_BENCH_STEP * args.steps * world
    value = ion_steps / (ms_max * 1e-3)

    # roofline of the dominant (fused step) kernel: algorithmic bytes per launch / mean launch duration
    peaks = measured_peaks()
    avg_launch_ms = kernel_ms / max(timed_launches, 1)
    bpl = BYTES_PER_ION_LAUNCH[args.precision] * n_ions
    achieved = bpl / (avg_launch_ms * 1e-3) / 1e9

    # The fused kernel moves the state through HBM once per 1000 steps, so
    # it is bound by instruction issue; its roofline leads with the issue
    # bound (from the ncu summary of the current kernel) and keeps the HBM
    # fraction beside it.
    prof = profile_figures(PROFILE_FUSED) if args.workload == "ims-1M" else {"fresh": False, "note": "not profiled"}
    kname = f"k_step<{args.precision},boris,hss,uniform> fused {sim_K(None)} steps/launch"
    hbm = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
           "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"], "bytes_per_launch": bpl,
           "traffic": prof.get("dram_bytes_per_launch") if args.steps_per_launch == 1000 else None}
    issue = issue_roofline(args, avg_launch_ms, clk, prof)
    if issue is not None:
        roofline = {**issue, "traffic": hbm["traffic"], "traffic_unit": "DRAM bytes per launch (ncu)",
                    "kernel": kname, "avg_launch_ms": avg_launch_ms, "hbm": hbm, "profile": prof}
    else:
        roofline = {**hbm, "traffic_unit": "DRAM bytes per launch (ncu)", "kernel": kname,
                    "avg_launch_ms": avg_launch_ms, "profile": prof,
                    "note": "issue roofline needs a current ncu summary of this kernel"}

    # The per-step kernel (collision_test = PER_STEP: one engine step per
    # launch, the state through HBM every step) on the same physics with
    # N_PER_STEP ions, so that the state (37 B per ion in the float forms)
    # is 5x the L2 and every launch streams it from HBM.  Algorithmic bytes
    # per ion-step: positions 24 + velocities 12 (24 in FP64) + flag 1 read,
    # positions and velocities written.
    per_step = None
    if args.workload == "ims-1M" and args.per_step_ions > 0:
        n1 = args.per_step_ions
        spec1 = cfg.species_spec(n1, 200.0 * cfg.AMU_TO_KG, cfg.ELEM_CHARGE_C,
                                 {"type": "gaussian", "center": [0, 0, 0], "std": [5e-4] * 3},
                                 {"type": "thermal", "temperature_K": 300.0})
        st1 = generate_ions(123, [spec1])
        b1 = {"fp64": 97, "mixed": 73, "hilo": 73}[args.precision]
        sim1 = Simulation(ensembles, precision=prec_id, integrator=capi.INTEGRATOR_BORIS,
                          collision=capi.COLLISION_HSS, rng_seed=123, device=dev,
                          collision_test=capi.TEST_PER_STEP)
        sim1.set_stream(stream.cuda_stream)
        sim1.upload(st1, first_id=first_id)
        del st1
        sim1.advance(10)
        torch.cuda.synchronize()
        n_launch = 40
        r1 = sim1.advance(n_launch)
        torch.cuda.synchronize()
        avg1 = r1["step_kernel_ms"] / n_launch
        ach1 = b1 * n1 / (avg1 * 1e-3) / 1e9
        sim1.close()
        prof1 = (profile_figures(PROFILE_STEP1, unit="icb_step1_mixed.cu")
                 if args.precision == "mixed" and n1 == 16 * 1048576 else {"fresh": False, "note": "not profiled"})
        per_step = {"bound": "hbm", "achieved": ach1, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": ach1 / peaks["hbm_gbs"], "peak_source": peaks["source"], "avg_launch_ms": avg1,
                    "kernel": f"k_step1_ws<{args.precision},hss> (collision_test = PER_STEP), 1 step/launch",
                    "ions": n1, "bytes_per_ion_step": b1, "bytes_per_launch": b1 * n1, "launches_timed": n_launch,
                    "traffic": prof1.get("dram_bytes_per_launch"), "traffic_unit": "DRAM bytes per launch (ncu)",
                    "profile": prof1, "ion_steps_per_s": n1 / (avg1 * 1e-3),
                    "collision_fraction": r1["collisions"] / (n1 * n_launch)}

    # The same workload in the other precision forms, each on a shorter
    # timed run, labelled by algorithm: the event-to-event drift (the
    # headline's algorithm) and the step-by-step loop in every precision, and
    # the reference's per-step algorithm (a Maxwell-Boltzmann neutral and an
    # exp test for every ion every step) in FP64.
    forms = None
    if args.precision == "mixed" and args.stepping == "events" and args.fp64_steps > 0:
        def time_form(prec, stepping, n_timed, collision=capi.COLLISION_HSS):
            sf = make_sim(prec, collision=collision, stepping=stepping)
            sf.advance(STEPS_PER_BENCH_STEP)
            sf.upload(st0, ens_offsets=offsets, first_id=first_id)
            torch.cuda.synchronize()
            msf, _, _, _, _ = timed_loop(sf, n_timed, STEPS_PER_BENCH_STEP, allreduce=False)
            sf.close()
            msf = parallel.max_over_ranks(msf)
            return {"value": n_ions * STEPS_PER_BENCH_STEP * n_timed * world / (msf * 1e-3), "unit": "ion-steps/s",
                    "steps": n_timed}
        nf = args.fp64_steps
        forms = {
            "mixed_events": {"value": value, "unit": "ion-steps/s", "steps": args.steps,
                             "form": "f32 v / f64 x, event-to-event drift (the headline)"},
            "hilo_events": {**time_form(capi.PREC_MIXED_HILO, capi.STEPPING_EVENTS, nf),
                            "form": "f32 v / compensated f32 hi-lo x, event-to-event drift"},
            "fp64_events": {**time_form(capi.PREC_FP64, capi.STEPPING_EVENTS_ALL, nf),
                            "form": "f64, event-to-event drift (same algorithm as the headline)"},
            "mixed_per_step": {**time_form(capi.PREC_MIXED, capi.STEPPING_PER_STEP, nf),
                               "form": "f32 v / f64 x, step-by-step loop with deferred collisions"},
            "fp64_per_step": {**time_form(capi.PREC_FP64, capi.STEPPING_PER_STEP, nf),
                              "form": "f64, step-by-step loop (same algorithm as mixed_per_step; the "
                                      "bit-faithful FP64 form of the parity tests)"},
            "plain_fp64": {**time_form(capi.PREC_FP64, capi.STEPPING_PER_STEP, max(1, min(nf, 3)),
                                       collision=capi.COLLISION_HSS_PLAIN),
                           "form": "f64, the reference's per-step HSS algorithm (MB neutral + exp test "
                                   "every ion every step) with Philox: the plain FP64 GPU form"},
        }
        forms["speedups"] = {
            "precision_only_events": value / forms["fp64_events"]["value"],
            "precision_only_per_step": forms["mixed_per_step"]["value"] / forms["fp64_per_step"]["value"],
            "hilo_over_fp64_events": forms["hilo_events"]["value"] / forms["fp64_events"]["value"],
            "algorithm_and_precision_vs_plain_fp64": value / forms["plain_fp64"]["value"],
            "algorithm_only_fp64_events_vs_plain": forms["fp64_events"]["value"] / forms["plain_fp64"]["value"],
        }

    # end to end through the C ABI with host buffers: H2D state from pinned
    # memory, advance one snapshot interval, D2H state, every step
    e2e_steps = min(args.steps, args.e2e_steps)
    pin = {k: torch.empty(n_ions, dtype=torch.float64, pin_memory=True).numpy() for k in ("x", "y", "z", "vx", "vy", "vz")}
    pin_act = torch.empty(n_ions, dtype=torch.uint8, pin_memory=True).numpy()
    for k in pin:
        pin[k][:] = getattr(st0, k)
    pin_act[:] = 1
    host = IonState(x=pin["x"], y=pin["y"], z=pin["z"], vx=pin["vx"], vy=pin["vy"], vz=pin["vz"], mass=st0.mass,
                    charge=st0.charge, active=pin_act, t_death=None, t_arrival=None)
    sim.upload(st0, ens_offsets=offsets, first_id=first_id)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    # the host fast path overlaps each ion chunk's copies with the others' steps
    if args.e2e_chunks is None:
        args.e2e_chunks = 10 if args.workload == "en-sweep" else 24
    sim.advance_host(host, STEPS_PER_BENCH_STEP, n_chunks=args.e2e_chunks)      # warm the copy stream
    sim.upload(st0, ens_offsets=offsets, first_id=first_id)
    for k in pin:
        pin[k][:] = getattr(st0, k)
    pin_act[:] = 1
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.advance_host(host, STEPS_PER_BENCH_STEP, n_chunks=args.e2e_chunks)
    torch.cuda.synchronize()
    e2e_s = parallel.max_over_ranks(time.perf_counter() - t0)
    e2e_value = n_ions * STEPS_PER_BENCH_STEP * e2e_steps * world / e2e_s
    sim.close()

    # the CPU sample is the single-ensemble IMS workload; no CPU line for the sweep
    cpu = (cpu_baseline() if (rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "ims-1M")
           else None)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "ion-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"mixed": "f32 (v, field, collisions) + f64 (x, t)", "fp64": "f64",
                                       "hilo": "f32 (v) + f32 hi/lo (x)"}[args.precision],
        "data": "synthetic (reference ion-loader semantics, seed 123)",
        "config": {"workload": workload, "ions_per_gpu": n_ions, "engine_steps_per_bench_step": STEPS_PER_BENCH_STEP,
                   "total_engine_steps": STEPS_PER_BENCH_STEP * args.steps, "precision": args.precision,
                   "steps_per_launch": sim_K(None), "collisions": "HSS null-collision, Philox4x32-10",
                   "parallelism": f"ions sharded, {world} GPU(s)", "l2": "flushed between timed steps (256 MB write)",
                   "collision_fraction": stt["collisions"] / max(ion_steps / world, 1),
                   "cuda_graphs": bool(args.graphs), "autotuned": tuning, "stepping": args.stepping},
        "gpu_launches": launches,
        "roofline": roofline,
        "roofline_per_step": per_step,
        "precision_forms": forms,
        "e2e": {"value": e2e_value, "unit": "ion-steps/s", "h2d_bytes_per_step": 6 * 8 * n_ions,
                "d2h_bytes_per_step": 6 * 8 * n_ions + n_ions, "steps": e2e_steps,
                "path": f"icb_advance_host(1000 steps, {args.e2e_chunks} ion chunks): pinned host state in and out, "
                        "copies of each chunk overlapped with the steps of the others"},
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


def run_fticr(args) -> None:
    """FT-ICR cell with space charge (262,144 ions, P3M on a 128^3 mesh, one
    solve per engine step): ion-steps/s of the whole step and the P3M solve
    time per step.  Under torchrun the cell's ions are sharded over the ranks
    (strong scaling): before every step each rank exports its ions, an NCCL
    all-gather gives every rank all of them, and each rank's solve deposits
    and pairs with every ion but computes the field of its own.

    The push runs in FP64 by default: at 2.7 km/s on the cyclotron orbit the
    trap field's kick per half step (|q E / m| dt / 2 ~ 2e-4 m/s at m/z 500)
    is below one float ulp of the velocity (2.4e-4 m/s), so the float
    velocity of the mixed form rounds the magnetron part of the motion and
    shifts w+ by a few ppm.  The P3M mesh stays in single precision (its
    field is resolution-limited at ~2 % RMS); --sc-solver-fp64 runs it in
    FP64."""
    import torch

    sys.path.insert(0, str(ROOT))
    from icarion_b200 import _capi as capi
    from icarion_b200 import fticr, parallel
    from icarion_b200.sim import IonState, Simulation

    rank, world, local = _env_rank()
    torch.cuda.set_device(local if world > 1 else 0)
    dev = torch.cuda.current_device()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    prec_id = {"mixed": capi.PREC_MIXED, "fp64": capi.PREC_FP64}[args.precision if args.precision != "hilo" else "mixed"]
    cell = fticr.fticr_cell()
    n = cell.ions.n
    b, e = parallel.shard_range(n, rank, world)
    mine = IonState(**{k: np.ascontiguousarray(getattr(cell.ions, k)[b:e])
                       for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "charge", "active")},
                    t_death=None, t_arrival=None)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    steps_per = 100
    sim = Simulation([cell.ensemble], precision=prec_id, integrator=capi.INTEGRATOR_BORIS,
                     collision=capi.COLLISION_LANGEVIN, rng_seed=123, device=dev,
                     use_graphs=int(args.graphs and world == 1))
    sim.set_stream(stream.cuda_stream)
    sim.upload(mine, first_id=b)
    solver_fp32 = prec_id != capi.PREC_FP64 or not args.sc_solver_fp64
    fticr.configure(sim, cell, solver_fp32=solver_fp32)
    exchange = parallel.SpaceChargeExchange(sim, e - b, (n + world - 1) // world) if world > 1 else None

    def advance(k: int) -> dict:
        if exchange is None:
            return sim.advance(k)
        tot = {}
        for _ in range(k):
            exchange.step()
            rs1 = sim.advance(1)
            for key, val in rs1.items():
                tot[key] = tot.get(key, 0) + val
        return tot

    for _ in range(args.warmup):
        advance(steps_per)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(dev)).split(",")[0]) if world == 1 else dev)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sc_ms, sc_n, step_ms, step_n, launches = 0.0, 0, 0.0, 0, 0
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        rs = advance(steps_per)
        ev[i][1].record(stream)
        sc_ms += rs["spacecharge_ms"]
        sc_n += rs["spacecharge_solves_timed"]
        step_ms += rs["step_kernel_ms"]
        step_n += min(steps_per, 64) if exchange is None else steps_per
        launches += rs["kernel_launches"]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b_) for a, b_ in ev)
    if world > 1:
        ms = parallel.max_over_ranks(ms)
    value = n * steps_per * args.steps / (ms * 1e-3)
    # solves are timed one by one only outside CUDA graphs
    p3m_ms = sc_ms / sc_n if sc_n else None
    # algorithmic HBM bytes of one isolated P3M solve on the (2*128)^3 grid,
    # each pass reading and writing its data once.  FP64 mesh (3D
    # transforms): deposit write, forward FFT read+write, 3 x (kernel
    # multiply: 2 reads + 1 write, inverse FFT read+write) of the real (8 B)
    # and half-complex (16 B x (M/2+1)/M) grids.  Single-precision mesh
    # (4 B; transforms pruned to the mesh planes x < M/2, the x pass fused
    # with the kernel products at M = 256): deposit write of the mesh
    # planes, their 2D (y, z) R2C, the fused x pass (their spectrum and the
    # folded kernel quadrants read, three components' mesh planes written)
    # and the three components' 2D C2R.  Plus per ion position/charge reads,
    # keys and the 8-node x 3-component gather.
    M = 2 * cell.sc_grid[0]
    esz = 4.0 if solver_fp32 else 8.0
    real_b = esz * M ** 3
    cplx_b = 2 * esz * M * M * (M // 2 + 1)
    if solver_fp32:
        fold_b = 3 * esz * (M // 2 + 1) ** 3
        grid_bytes = (real_b / 2 + (real_b / 2 + cplx_b / 2) + (cplx_b / 2 + fold_b + 3 * cplx_b / 2)
                      + 3 * (cplx_b / 2 + real_b / 2))
    else:
        grid_bytes = real_b + (real_b + cplx_b) + 3 * (3 * cplx_b) + 3 * (cplx_b + real_b)
    ion_bytes = n * (33 + 32 + 24 + 192 + 24)
    p3m_bytes = grid_bytes + ion_bytes
    achieved = p3m_bytes / (p3m_ms * 1e-3) / 1e9 if p3m_ms else None
    peaks = measured_peaks()
    # end to end: host state in, steps_per steps, host state out, per bench step
    e2e_steps = min(args.steps, args.e2e_steps)
    host = sim.download()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sim.update_state(host)
        advance(steps_per)
        sim.download(into=host)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        e2e_s = parallel.max_over_ranks(e2e_s)
    sim.close()
    if world > 1:
        del exchange
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    n_own = e - b
    line = {
        "metric": METRIC, "value": value, "unit": "ion-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak",
        "vs_baseline": None, "dtype": {capi.PREC_MIXED: "f32 (v, field) + f64 (x, t, space charge)",
                                       capi.PREC_FP64: "f64"}[prec_id] + (" (P3M mesh f32)" if solver_fp32 else ""),
        "data": "synthetic (reference ion-loader semantics, seed 123; m/z uniform 500-1500)",
        "config": {"workload": "FT-ICR cell, 262,144 ions (+1, m/z 500-1500), 7 T, 1 V quadrupolar trap, "
                               "He 1e-7 Pa Langevin capture, Boris dt 1e-9 s, P3M space charge 128^3 CIC "
                               "(isolated, 2-cell particle-particle cutoff) solved every step",
                   "ions_per_gpu": n_own, "engine_steps_per_bench_step": steps_per, "precision": args.precision,
                   "parallelism": (f"ions sharded over {world} GPUs, NCCL all-gather of every ion's (x, y, z, q) "
                                   "before each step, mesh solve on every rank, gather of own ions")
                                  if world > 1 else "1 GPU",
                   "l2": "flushed between timed steps",
                   "cuda_graphs": bool(args.graphs and world == 1), "p3m_ms_per_step": p3m_ms,
                   "push_ms_per_step": step_ms / max(step_n, 1)},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"] if achieved else None, "traffic": None,
                     "peak_source": peaks["source"],
                     "kernel": "isolated P3M solve (bin, sort, deposit, FFTs, kernel multiplies, gather + PP)",
                     "bytes_per_solve": p3m_bytes},
        "e2e": {"value": n * steps_per * e2e_steps / e2e_s, "unit": "ion-steps/s",
                "h2d_bytes_per_step": (6 * 8 * n_own + n_own) * world,
                "d2h_bytes_per_step": (6 * 8 * n_own + n_own + 2 * 8 * n_own) * world, "steps": e2e_steps},
        "clocks": clk,
        "cpu_baseline": None,
        "cpu_baseline_note": "the reference's CPU space charge is an O(N^2) direct sum; no bounded sample of this "
                             "workload is timed",
    }
    print(json.dumps(line))


def run_ipm(args) -> None:
    """Learned interaction-potential collisions: train the deflection network
    on 2^20 quadrature samples, then advance 1,048,576 ions of 300 Da in N2
    (three ensembles at 10, 40 and 80 Td) with the table and with the
    network, reporting ion-steps/s of both and their K0."""
    import torch

    sys.path.insert(0, str(ROOT))
    from icarion_b200 import _capi as capi
    from icarion_b200 import config as cfg
    from icarion_b200 import ipm
    from icarion_b200.sim import Simulation

    rank, world, local = _env_rank()
    torch.cuda.set_device(local if world > 1 else 0)
    dev = torch.cuda.current_device()
    setup = ipm.IpmSetup()
    t0 = time.perf_counter()
    x, y, _, _ = ipm.training_set(setup, n=1 << 20, seed=2024, device=dev)
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    params, losses = ipm.train(x, y, epochs=20, batch=1024, lr=3e-3, seed=7, device=dev)
    t_train = time.perf_counter() - t0
    xv, yv, _, _ = ipm.training_set(setup, n=1 << 16, seed=99, device=dev)
    val_rms = float(np.sqrt(np.mean((ipm.forward(params, xv, mode=1, device=dev) - yv) ** 2)))

    en = (10.0, 40.0, 80.0)
    n_total = N_IONS
    ensembles, st0, offsets = ipm.drift_ensembles(setup, en, n_total)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    results = {}
    launches = 0
    clocks = ClockSampler(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(dev)).split(",")[0]) if world == 1 else dev)
    clocks.start()
    # the table, the learned network, and the FP64 quadrature at every
    # collision (the method without the network; timed on fewer steps)
    for name, model in (("table", capi.COLLISION_IPM_TABLE), ("mlp", capi.COLLISION_IPM_MLP),
                        ("quadrature", capi.COLLISION_IPM_QUAD)):
        n_timed = args.steps if model != capi.COLLISION_IPM_QUAD else min(args.steps, 2)
        sim = Simulation(ensembles, precision=capi.PREC_MIXED, collision=model, rng_seed=123, device=dev,
                         stepping=STEPPING[args.stepping])
        sim.set_stream(stream.cuda_stream)
        sim.upload(st0, ens_offsets=offsets, first_id=rank * n_total)
        sim.configure_ipm(setup)
        if model == capi.COLLISION_IPM_MLP:
            sim.set_mlp(params)
        tuned = sim.autotune(300) if args.autotune and model != capi.COLLISION_IPM_QUAD else None
        for _ in range(args.warmup if model != capi.COLLISION_IPM_QUAD else 1):
            sim.advance(STEPS_PER_BENCH_STEP)
        sim.upload(st0, ens_offsets=offsets, first_id=rank * n_total)
        sim.set_clock(0, np.zeros(3))
        torch.cuda.synchronize()
        ms, kms, nl, coll = 0.0, 0.0, 0, 0
        for _ in range(n_timed):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            rs = sim.advance(STEPS_PER_BENCH_STEP)
            b.record(stream)
            torch.cuda.synchronize()
            ms += a.elapsed_time(b)
            kms += rs["step_kernel_ms"]
            nl += rs["kernel_launches"]
            coll += rs["collisions"]
        launches += nl
        mom = sim.moments()
        _, tcl = sim.clock()
        k0 = []
        for e in range(3):
            dz = mom[e][16] / mom[e][0]
            v_d = dz / tcl[e]
            n_gas = ensembles[e]["gas_density_m3"]
            E = en[e] * 1e-21 * n_gas
            k0.append(v_d / E * (n_gas / cfg.n0_loschmidt()) * 1e4)
        results[name] = {"autotuned": tuned,
                         "ion_steps_per_s": n_total * STEPS_PER_BENCH_STEP * n_timed / (ms * 1e-3),
                         "ms_per_step": ms / n_timed, "K0_cm2_Vs": k0, "timed_steps": n_timed,
                         "collision_fraction": coll / (n_total * STEPS_PER_BENCH_STEP * n_timed)}
        sim.close()
    clk = clocks.stop()
    if rank != 0:
        return
    peaks = measured_peaks()
    mlp = results["mlp"]
    bpl = BYTES_PER_ION_LAUNCH["mixed"] * n_total
    achieved = bpl / (mlp["ms_per_step"] * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": mlp["ion_steps_per_s"], "unit": "ion-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": mlp["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (v, field, collisions) + bf16 MMA (network) + f64 (x, t)",
        "data": "synthetic (reference ion-loader semantics, seed 123; training pairs seed 2024)",
        "config": {"workload": "learned interaction-potential collisions: LJ 12-6 (5 meV, r_m 4 A) + C4 "
                               "(N2 1.74 A^3) ion-N2 potential, 300 Da, 1,048,576 ions in three ensembles at "
                               "10/40/80 Td, N2 300 K 1000 Pa, b_max 12 A, dt = 0.1/nu_max",
                   "ions_per_gpu": n_total, "engine_steps_per_bench_step": STEPS_PER_BENCH_STEP,
                   "table": results["table"], "mlp": mlp, "quadrature": results["quadrature"],
                   "K0_shift_mlp_vs_table": [m / t - 1.0 for m, t in zip(mlp["K0_cm2_Vs"], results["table"]["K0_cm2_Vs"])],
                   "speedup_mlp_over_quadrature": mlp["ion_steps_per_s"] / results["quadrature"]["ion_steps_per_s"],
                   "speedup_mlp_over_table": mlp["ion_steps_per_s"] / results["table"]["ion_steps_per_s"],
                   "K0_note": "K0 here is <dz>/t over the timed steps (transient included); the K0 gates are "
                              "fitted in tests/test_gpu_ipm_config3.py",
                   "training": {"samples": 1 << 20, "epochs": 20, "batch": 1024, "data_s": t_data,
                                "train_s": t_train, "final_loss": float(losses[-1]),
                                "validation_rms_cos_chi": val_rms},
                   "l2": "flushed between timed steps"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": None, "peak_source": peaks["source"],
                     "kernel": "k_step<mixed,boris,ipm-mlp,uniform> fused 1000 steps/launch",
                     "note": "state crosses HBM once per 1000-step launch: issue bound, not HBM bound"},
        "e2e": None,
        "clocks": clk,
        "cpu_baseline": None,
        "cpu_baseline_note": "the reference's IPM handler needs its HDF5 offline tables (not buildable here)",
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64", "hilo"], default=None,
                    help="default mixed; fticr-sc: fp64 (the float velocity biases the cyclotron frequency)")
    ap.add_argument("--sc-solver-fp64", action="store_true",
                    help="fticr-sc under fp64: run the P3M mesh in FP64 too (default single precision)")
    ap.add_argument("--steps-per-launch", type=int, default=1000)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--pending", type=int, default=0)
    ap.add_argument("--spv", type=int, default=0, help="collision-free steps between warp votes")
    ap.add_argument("--stepping", choices=["events", "per-step", "events-all"], default="events",
                    help="float forms: event-to-event closed-form drift, or the step-by-step loop")
    ap.add_argument("--workload", choices=["ims-1M", "en-sweep", "fticr-sc", "ipm", "tims-1M"], default="ims-1M",
                    help="ims-1M: the 1,048,576-ion IMS run (default); en-sweep: the batched 64-ensemble E/N "
                         "sweep; fticr-sc: the 262,144-ion FT-ICR cell with P3M space charge; ipm: learned "
                         "interaction-potential collisions vs the table")
    ap.add_argument("--autotune", action="store_true", help="pick the launch shape with icb_autotune first")
    ap.add_argument("--graphs", action="store_true", help="replay icb_advance through CUDA graphs")
    ap.add_argument("--fp64-steps", type=int, default=10)
    ap.add_argument("--per-step-ions", type=int, default=16 * 1048576,
                    help="ions of the per-step kernel's HBM roofline run (0 = skip)")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--e2e-chunks", type=int, default=None,
                    help="ion chunks of the overlapped host path (default: 24 for ims-1M, whose steps outlast "
                         "the copies; 10 for en-sweep, whose copies outlast the steps and whose chunks then "
                         "pay their per-chunk host calls)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.precision is None:
        args.precision = "fp64" if args.workload == "fticr-sc" else "mixed"
    if args.warmup < 3 and args.impl == "ours":
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "fticr-sc":
        run_fticr(args)
    elif args.workload == "ipm":
        run_ipm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
