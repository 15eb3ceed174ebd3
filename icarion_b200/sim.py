"""Host mirror of the reference's batch-step plug points over the C ABI.

``Simulation`` owns one ``icb_handle``: the device-resident ion SoA plus the
per-ensemble constants.  It exposes the reference's call pattern:

* ``step_batch(t, dt)``  -> IIntegrationStrategy::step_batch (push only)
* ``handle_batch(dt)``   -> ICollisionHandler::handle_batch (collisions only)
* ``finalize()``         -> SimulationEngine::finalize_ions_after_integration
* ``advance(n)``         -> n fused engine steps (SimulationEngine::process_timestep)

and ``run(n_steps, write_interval)`` for the engine's snapshot loop.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from . import config as cfgmod


@dataclass
class IonState:
    """IonEnsemble hot/cold SoA arrays (IonEnsemble.h:267-330) on the host."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    mass: np.ndarray
    charge: np.ndarray
    active: np.ndarray
    birth: np.ndarray | None = None
    t_death: np.ndarray | None = None
    t_arrival: np.ndarray | None = None

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def copy(self) -> "IonState":
        return IonState(**{k: (None if v is None else np.array(v, copy=True)) for k, v in self.__dict__.items()})

    @staticmethod
    def empty(n: int) -> "IonState":
        z = lambda: np.zeros(n, dtype=np.float64)  # noqa: E731
        return IonState(z(), z(), z(), z(), z(), z(), z(), z(), np.ones(n, dtype=np.uint8),
                        None, np.full(n, -1.0), np.full(n, -1.0))

    @staticmethod
    def concat(states: list["IonState"]) -> "IonState":
        out = {}
        for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "charge", "active"):
            out[k] = np.ascontiguousarray(np.concatenate([getattr(s, k) for s in states]))
        n = sum(s.n for s in states)
        out["t_death"] = np.full(n, -1.0)
        out["t_arrival"] = np.full(n, -1.0)
        return IonState(**out)


def generate_ions(rng_seed: int, specs: list[capi.SpeciesSpec]) -> IonState:
    """Initial cloud with the reference IonLoader semantics (host C++)."""
    n = sum(int(s.count) for s in specs)
    st = IonState.empty(n)
    arr = (capi.SpeciesSpec * len(specs))(*specs)
    capi.check(capi.lib().icb_generate_ions(
        C.c_uint32(rng_seed & 0xFFFFFFFF), len(specs), arr,
        capi.dptr(st.x), capi.dptr(st.y), capi.dptr(st.z), capi.dptr(st.vx), capi.dptr(st.vy), capi.dptr(st.vz),
        capi.dptr(st.mass), capi.dptr(st.charge)))
    return st


def device_count() -> int:
    c = C.c_int(0)
    rc = capi.lib().icb_device_count(C.byref(c))
    return c.value if rc == 0 else 0


class Simulation:
    """One device-resident population of ions in one or more ensembles.

    The keyword arguments are the fields of ``icb_config``: ``precision``
    (PREC_FP64 / PREC_MIXED / PREC_MIXED_HILO), ``integrator``, ``collision``
    (COLLISION_*), ``rng_seed``, ``device``; launch shape ``block_size``,
    ``steps_per_launch``, ``pending_threshold``, ``steps_per_vote`` (0 =
    defaults), ``use_graphs``; ``stepping`` (STEPPING_EVENTS: the float forms
    move each ion from event to event in closed form; STEPPING_PER_STEP: the
    step-by-step loop); ``collision_subcycles`` (collision tests per step,
    plain FP64 form only); ``collision_test`` (TEST_CLOCK: the collision clock
    of the fused kernels; TEST_PER_STEP: the stateless per-step test of the
    per-step kernel).
    """

    def __init__(self, ensembles: list[dict], precision: int = capi.PREC_MIXED,
                 integrator: int = capi.INTEGRATOR_BORIS, collision: int = capi.COLLISION_HSS,
                 rng_seed: int = 123, device: int = 0, block_size: int = 0, steps_per_launch: int = 0,
                 pending_threshold: int = 0, use_graphs: int = 0, steps_per_vote: int = 0,
                 stepping: int = capi.STEPPING_EVENTS, collision_subcycles: int = 0,
                 collision_test: int = capi.TEST_CLOCK):
        self._lib = capi.lib()
        self.n_ens = len(ensembles)
        self._ens = (capi.EnsembleParams * self.n_ens)(*[cfgmod.to_struct(e) for e in ensembles])
        cfg = capi.Config()
        cfg.precision = precision
        cfg.integrator = integrator
        cfg.collision_model = collision
        cfg.n_ensembles = self.n_ens
        cfg.ensembles = C.cast(self._ens, C.POINTER(capi.EnsembleParams))
        cfg.rng_seed = rng_seed
        cfg.device = device
        cfg.block_size = block_size
        cfg.steps_per_launch = steps_per_launch
        cfg.pending_threshold = pending_threshold
        cfg.use_graphs = use_graphs
        cfg.steps_per_vote = steps_per_vote
        cfg.stepping = stepping
        cfg.collision_subcycles = collision_subcycles
        cfg.collision_test = collision_test
        self._h = C.c_void_p()
        capi.check(self._lib.icb_create(C.byref(cfg), C.byref(self._h)))
        self.ensembles = ensembles
        self.precision = precision
        self.n = 0

    # -- lifetime ------------------------------------------------------------
    def close(self) -> None:
        if self._h:
            self._lib.icb_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ---------------------------------------------------------------
    def upload(self, st: IonState, ens_offsets: np.ndarray | None = None, first_id: int = 0) -> None:
        off = None if ens_offsets is None else np.ascontiguousarray(ens_offsets, dtype=np.uint64)
        capi.check(self._lib.icb_upload_ions(
            self._h, st.n, capi.dptr(st.x), capi.dptr(st.y), capi.dptr(st.z),
            capi.dptr(st.vx), capi.dptr(st.vy), capi.dptr(st.vz), capi.dptr(st.mass), capi.dptr(st.charge),
            capi.u8ptr(st.active), capi.dptr(st.birth), capi.u64ptr(off), first_id))
        self.n = st.n

    def update_state(self, st: IonState) -> None:
        capi.check(self._lib.icb_update_state(
            self._h, capi.dptr(st.x), capi.dptr(st.y), capi.dptr(st.z),
            capi.dptr(st.vx), capi.dptr(st.vy), capi.dptr(st.vz), capi.u8ptr(st.active)))

    def download(self, into: IonState | None = None) -> IonState:
        st = into if into is not None else IonState.empty(self.n)
        if st.t_death is None:
            st.t_death = np.full(self.n, -1.0)
        if st.t_arrival is None:
            st.t_arrival = np.full(self.n, -1.0)
        capi.check(self._lib.icb_download_ions(
            self._h, capi.dptr(st.x), capi.dptr(st.y), capi.dptr(st.z),
            capi.dptr(st.vx), capi.dptr(st.vy), capi.dptr(st.vz), capi.u8ptr(st.active),
            capi.dptr(st.t_death), capi.dptr(st.t_arrival)))
        return st

    # -- stepping -------------------------------------------------------------
    def advance(self, n_steps: int) -> dict:
        rs = capi.RunStats()
        capi.check(self._lib.icb_advance(self._h, int(n_steps), C.byref(rs)))
        return rs.as_dict()

    def advance_host(self, st: IonState, n_steps: int, n_chunks: int = 24) -> dict:
        """Host state in, n_steps, host state out (positions, velocities and
        active flags of ``st`` are read and overwritten), copies overlapped
        with the steps of other ion chunks (icb_advance_host)."""
        rs = capi.RunStats()
        capi.check(self._lib.icb_advance_host(
            self._h, int(n_steps), int(n_chunks), capi.dptr(st.x), capi.dptr(st.y), capi.dptr(st.z),
            capi.dptr(st.vx), capi.dptr(st.vy), capi.dptr(st.vz), capi.u8ptr(st.active), C.byref(rs)))
        return rs.as_dict()

    def advance_async(self, n_steps: int) -> None:
        capi.check(self._lib.icb_advance(self._h, int(n_steps), None))

    def step_batch(self) -> bool:
        """IIntegrationStrategy::step_batch: push every active ion once."""
        capi.check(self._lib.icb_push(self._h))
        return True

    def handle_batch(self) -> dict:
        """ICollisionHandler::handle_batch: one collision test per active ion."""
        rs = capi.RunStats()
        capi.check(self._lib.icb_collide(self._h, C.byref(rs)))
        return rs.as_dict()

    def finalize(self) -> dict:
        rs = capi.RunStats()
        capi.check(self._lib.icb_finalize(self._h, C.byref(rs)))
        return rs.as_dict()

    def synchronize(self) -> None:
        capi.check(self._lib.icb_synchronize(self._h))

    def set_stream(self, stream_ptr: int | None) -> None:
        capi.check(self._lib.icb_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def clock(self) -> tuple[int, np.ndarray]:
        st = C.c_uint64(0)
        t = np.zeros(self.n_ens)
        capi.check(self._lib.icb_get_clock(self._h, C.byref(st), capi.dptr(t)))
        return st.value, t

    def set_clock(self, step: int, t: np.ndarray) -> None:
        t = np.ascontiguousarray(t, dtype=np.float64)
        capi.check(self._lib.icb_set_clock(self._h, int(step), capi.dptr(t)))

    def moments(self) -> np.ndarray:
        out = np.zeros((self.n_ens, capi.N_MOMENTS))
        capi.check(self._lib.icb_moments(self._h, capi.dptr(out)))
        return out

    def mark_reference(self) -> None:
        capi.check(self._lib.icb_mark_reference(self._h))

    def configure_space_charge(self, mode: int, grid_n, box_min, box_max, alpha_h: float = 0.0,
                               pp_cutoff_cells: float = 0.0, softening_m: float = -1.0,
                               field_bound: float = 0.0, solver_fp32: bool = False) -> None:
        """Space charge solved before every step (see icb_spacecharge_configure);
        solver_fp32 runs the isolated solver in single precision under an
        FP64 handle too."""
        c = capi.SpaceChargeConfig()
        c.mode = mode
        c.grid_n[:] = [int(v) for v in grid_n]
        c.box_min_m[:] = [float(v) for v in box_min]
        c.box_max_m[:] = [float(v) for v in box_max]
        c.alpha_h = alpha_h
        c.pp_cutoff_cells = pp_cutoff_cells
        c.softening_m = softening_m
        c.field_bound_V_m = field_bound
        c.solver_fp32 = 1 if solver_fp32 else 0
        capi.check(self._lib.icb_spacecharge_configure(self._h, C.byref(c)))

    def spacecharge_export(self, xyzq_device_ptr: int) -> None:
        """This handle's ions as (x, y, z, q) rows into a device buffer of
        n rows (see icb_spacecharge_export)."""
        capi.check(self._lib.icb_spacecharge_export(self._h, C.c_void_p(xyzq_device_ptr)))

    def set_spacecharge_peers(self, xyzq_device_ptr: int, n: int, skip_begin: int = 0, skip_count: int = 0) -> None:
        """Other devices' ions in this handle's solve (see
        icb_spacecharge_set_peers); n = 0 removes them."""
        capi.check(self._lib.icb_spacecharge_set_peers(self._h, int(n), C.c_void_p(xyzq_device_ptr or 0),
                                                       int(skip_begin), int(skip_count)))

    def space_charge_field(self) -> np.ndarray:
        """[3, n] space-charge field (V/m) of the current state."""
        out = np.zeros((3, self.n))
        capi.check(self._lib.icb_spacecharge_field(self._h, capi.dptr(out[0]), capi.dptr(out[1]),
                                                   capi.dptr(out[2])))
        return out

    def configure_ipm(self, setup) -> None:
        """Build the interaction-potential cos(chi) table (an ipm.IpmSetup)."""
        c = setup.config()
        capi.check(self._lib.icb_ipm_configure(self._h, C.byref(c)))
        self._ipm_shape = (setup.n_E, setup.n_b)

    def ipm_table(self) -> np.ndarray:
        out = np.zeros(self._ipm_shape, dtype=np.float32)
        capi.check(self._lib.icb_ipm_table(self._h, capi.fptr(out.reshape(-1))))
        return out

    def set_ehss_geometry(self, ensemble: int, centers_m: np.ndarray, radii_m: np.ndarray,
                          gas_radius_m: float) -> None:
        c = np.ascontiguousarray(centers_m, dtype=np.float64).reshape(-1, 3)
        r = np.ascontiguousarray(radii_m, dtype=np.float64)
        capi.check(self._lib.icb_ehss_set_geometry(self._h, ensemble, c.shape[0], capi.dptr(c.ravel()),
                                                   capi.dptr(r), gas_radius_m))

    def set_waveform(self, ensemble: int, channel: int, w: capi.Waveform | None) -> None:
        """Drive one field channel (capi.CHANNEL_*) of an ensemble by a
        waveform, or back to its constant (None)."""
        capi.check(self._lib.icb_set_waveform(self._h, ensemble, channel, C.byref(w) if w is not None else None))

    def set_tims_field(self, ensemble: int, f: capi.TimsField | None) -> None:
        """TIMS axial field of a TIMS ensemble (None: zero axial field)."""
        capi.check(self._lib.icb_set_tims_field(self._h, ensemble, C.byref(f) if f is not None else None))

    def apply_time_fields(self, ensemble: int, domain: dict, global_waveforms: dict | None = None) -> None:
        """Waveforms and TIMS field of a reference JSON domain
        (config.time_fields) on one ensemble."""
        waves, tims = cfgmod.time_fields(domain, global_waveforms)
        if tims is not None:
            self.set_tims_field(ensemble, tims)
        for ch, w in waves.items():
            self.set_waveform(ensemble, ch, w)

    def set_mlp(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        capi.check(self._lib.icb_ipm_set_mlp(self._h, capi.fptr(p)))

    def autotune(self, trial_steps: int = 0) -> dict:
        """Pick the fastest launch shape on the uploaded ions; the state and
        clock are restored, so the run continues unchanged (see icb_autotune)."""
        t = capi.Tuning()
        capi.check(self._lib.icb_autotune(self._h, trial_steps, C.byref(t)))
        return t.as_dict()

    def run(self, n_steps: int, write_interval: int, ref_step: int = 0,
            writer=None) -> tuple[np.ndarray, np.ndarray, dict]:
        """Advance n_steps, taking moments every write_interval steps (the
        engine's snapshot cadence).  Displacement moments are relative to the
        positions after ref_step steps (a multiple of write_interval).  With a
        ``snapshots.TrajectoryWriter`` every snapshot's state is also written
        (time of ensemble 0).  Returns (snapshot step indices, moments
        [snap, ens, 20], totals)."""
        if ref_step % write_interval:
            raise ValueError("ref_step must be a multiple of write_interval")
        steps, moms = [], []
        tot = {"candidates": 0, "collisions": 0, "rate_overflows": 0, "deaths": 0, "arrivals": 0, "device_ms": 0.0}
        done = 0
        while done < n_steps:
            k = min(write_interval, n_steps - done)
            rs = self.advance(k)
            for key in tot:
                tot[key] += rs[key]
            done += k
            if done == ref_step:
                self.mark_reference()
            steps.append(done)
            moms.append(self.moments())
            if writer is not None:
                writer.append(float(self.clock()[1][0]), self.download())
        return np.asarray(steps), np.stack(moms), tot
