"""ctypes bindings of the C ABI declared in include/icarion_b200.h.

The shared library is built in-tree (``icarion_b200/_lib/libicarion_b200.so``,
see ``icarion_b200.build``).  There is no CPU fallback: importing this module
without the library raises, and every entry point raises ``IcbError`` on a
non-zero status, like the reference's integrator/collision calls throw.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libicarion_b200.so"

ICB_OK = 0
ICB_ERR_INVALID_ARGUMENT = 1
ICB_ERR_CUDA = 2
ICB_ERR_OUT_OF_MEMORY = 3
ICB_ERR_UNSUPPORTED = 4
ICB_ERR_STATE = 5
ICB_ERR_NO_DEVICE = 6
ICB_ERR_TIMEOUT = 7

PREC_FP64, PREC_MIXED, PREC_MIXED_HILO = 0, 1, 2
INTEGRATOR_BORIS, INTEGRATOR_RK4 = 0, 1
COLLISION_NONE, COLLISION_HSS, COLLISION_IPM_TABLE, COLLISION_IPM_MLP, COLLISION_LANGEVIN = 0, 1, 2, 3, 4
COLLISION_HSS_PLAIN, COLLISION_EHSS, COLLISION_IPM_QUAD = 5, 6, 7
INSTRUMENT_IMS, INSTRUMENT_FTICR, INSTRUMENT_QUADRUPOLE_RF, INSTRUMENT_LQIT, INSTRUMENT_TIMS = 0, 1, 2, 3, 4
MAX_WAVE_POINTS = 64
(WAVE_CONSTANT, WAVE_LINEAR, WAVE_QUADRATIC, WAVE_EXPONENTIAL, WAVE_SINUSOIDAL, WAVE_PWM, WAVE_PULSED,
 WAVE_ARBITRARY) = range(8)
INTERP_LINEAR, INTERP_STEP, INTERP_CUBIC = 0, 1, 2
(CHANNEL_DC_AXIAL_V, CHANNEL_DC_QUAD_V, CHANNEL_RF_VOLTAGE_V, CHANNEL_RF_FREQUENCY_HZ,
 CHANNEL_TIMS_RAMP_FRACTION, CHANNEL_AC_X_AMPLITUDE_V, CHANNEL_AC_X_FREQUENCY_HZ, CHANNEL_AC_X_RAMP,
 CHANNEL_AC_Y_AMPLITUDE_V, CHANNEL_AC_Y_FREQUENCY_HZ, CHANNEL_AC_Y_RAMP, N_CHANNELS) = range(12)
TIMS_RAMP_LINEAR, TIMS_RAMP_EXPONENTIAL = 0, 1
SC_OFF, SC_P3M_ISOLATED, SC_PM_PERIODIC_REF = 0, 1, 2
STEPPING_EVENTS, STEPPING_PER_STEP, STEPPING_EVENTS_ALL = 0, 1, 2
TEST_CLOCK, TEST_PER_STEP = 0, 1
MATH_NEG_LOG1M, MATH_NEG_LOG1M_CUDA, MATH_ONE_MINUS_EXP, MATH_ONE_MINUS_EXP_CUDA = 0, 1, 2, 3
FLOW_CONSTANT, FLOW_AXIAL_UNIFORM, FLOW_AXIAL_PARABOLIC = 0, 1, 2
MLP_HIDDEN, MLP_N_PARAMS = 64, 4417
POS_POINT, POS_GAUSSIAN, POS_UNIFORM_SPHERE, POS_UNIFORM_CYLINDER, POS_UNIFORM_BOX = 0, 1, 2, 3, 4
VEL_FIXED, VEL_THERMAL = 0, 1
N_MOMENTS = 20
MAX_ENSEMBLES = 256

_ERR_NAMES = {
    1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "unsupported",
    5: "bad state", 6: "no CUDA device", 7: "timeout",
}


class IcbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"icarion_b200: {_ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


D3 = C.c_double * 3


class EnsembleParams(C.Structure):
    _fields_ = [
        ("instrument", C.c_int32), ("magnetic_enabled", C.c_int32),
        ("origin_m", D3), ("length_m", C.c_double), ("radius_m", C.c_double),
        ("axial_V", C.c_double), ("radial_V", C.c_double), ("dc_quad_V", C.c_double),
        ("rf_voltage_V", C.c_double), ("rf_frequency_Hz", C.c_double), ("B_T", D3),
        ("temperature_K", C.c_double), ("gas_density_m3", C.c_double), ("gas_mass_kg", C.c_double),
        ("gas_velocity_m_s", D3), ("gas_polarizability_m3", C.c_double), ("sigma_m2", C.c_double),
        ("ipm_bmax_m", C.c_double), ("dt_s", C.c_double), ("detector_z_m", C.c_double),
        ("n_gas", C.c_int32), ("flow_model", C.c_int32), ("gas_mix_density_m3", C.c_double * 8),
        ("gas_mix_mass_kg", C.c_double * 8), ("gas_mix_sigma_m2", C.c_double * 8),
        ("axial_flow_velocity_m_s", C.c_double), ("axial_flow_max_velocity_m_s", C.c_double),
        ("ac_amplitude_V", C.c_double * 2), ("ac_frequency_Hz", C.c_double * 2), ("ac_phase_rad", C.c_double * 2),
        ("ac_ramp", C.c_double * 2), ("ac_dipolar", C.c_int32), ("reserved2_", C.c_int32),
    ]


class Config(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("integrator", C.c_int32), ("collision_model", C.c_int32),
        ("n_ensembles", C.c_int32), ("ensembles", C.POINTER(EnsembleParams)), ("rng_seed", C.c_uint64),
        ("device", C.c_int32), ("block_size", C.c_int32), ("steps_per_launch", C.c_int32),
        ("pending_threshold", C.c_int32), ("use_graphs", C.c_int32), ("steps_per_vote", C.c_int32),
        ("stepping", C.c_int32), ("collision_subcycles", C.c_int32), ("collision_test", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


class RunStats(C.Structure):
    _fields_ = [
        ("steps", C.c_uint64), ("candidates", C.c_uint64), ("collisions", C.c_uint64),
        ("rate_overflows", C.c_uint64), ("deaths", C.c_uint64), ("arrivals", C.c_uint64),
        ("device_ms", C.c_double), ("step_kernel_ms", C.c_double), ("kernel_launches", C.c_uint64),
        ("spacecharge_ms", C.c_double), ("spacecharge_solves_timed", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Waveform(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("clamp", C.c_int32), ("interp", C.c_int32), ("n_points", C.c_int32),
        ("p", C.c_double * 8), ("times_s", C.c_double * 64), ("values", C.c_double * 64),
    ]


class TimsField(C.Structure):
    _fields_ = [
        ("ramp_mode", C.c_int32), ("n_nodes", C.c_int32), ("has_final_profile", C.c_int32),
        ("reserved_", C.c_int32), ("initial_uniform_V_m", C.c_double), ("final_uniform_V_m", C.c_double),
        ("ramp_start_s", C.c_double), ("ramp_end_s", C.c_double), ("ramp_tau_s", C.c_double),
        ("z_positions_m", C.c_double * 64), ("initial_profile_V_m", C.c_double * 64),
        ("final_profile_V_m", C.c_double * 64),
    ]


class SpaceChargeConfig(C.Structure):
    _fields_ = [
        ("mode", C.c_int32), ("grid_n", C.c_int32 * 3), ("box_min_m", D3), ("box_max_m", D3),
        ("alpha_h", C.c_double), ("pp_cutoff_cells", C.c_double), ("softening_m", C.c_double),
        ("field_bound_V_m", C.c_double), ("solver_fp32", C.c_int32), ("reserved", C.c_int32 * 7),
    ]


class IpmPotential(C.Structure):
    _fields_ = [("epsilon_J", C.c_double), ("r_m_m", C.c_double), ("polarizability_m3", C.c_double),
                ("charge_C", C.c_double)]


class IpmConfig(C.Structure):
    _fields_ = [("potential", IpmPotential), ("b_max_m", C.c_double), ("E_min_J", C.c_double),
                ("E_max_J", C.c_double), ("n_E", C.c_int32), ("n_b", C.c_int32), ("net_E_min_J", C.c_double),
                ("net_E_max_J", C.c_double), ("reserved", C.c_int32 * 2)]


class MlpTrainConfig(C.Structure):
    _fields_ = [("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_double), ("lr_min", C.c_double),
                ("seed", C.c_uint64), ("bf16_forward", C.c_int32), ("reserved", C.c_int32 * 5)]


class Tuning(C.Structure):
    _fields_ = [
        ("block_size", C.c_int32), ("steps_per_vote", C.c_int32), ("pending_threshold", C.c_int32),
        ("steps_per_launch", C.c_int32), ("trials", C.c_int32), ("reserved", C.c_int32),
        ("ion_steps_per_s", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class SpeciesSpec(C.Structure):
    _fields_ = [
        ("count", C.c_uint64), ("mass_kg", C.c_double), ("charge_C", C.c_double),
        ("position_type", C.c_int32), ("velocity_type", C.c_int32),
        ("center_m", D3), ("std_m", D3), ("radius_m", C.c_double), ("length_m", C.c_double),
        ("box_min_m", D3), ("box_max_m", D3), ("velocity_m_s", D3), ("temperature_K", C.c_double),
    ]


_P = C.POINTER
_DP = _P(C.c_double)
_FP = _P(C.c_float)
_U8P = _P(C.c_uint8)
_U32P = _P(C.c_uint32)
_U64P = _P(C.c_uint64)
_H = C.c_void_p

# name -> (restype, argtypes); every name here is declared in include/icarion_b200.h
SIGNATURES = {
    "icb_abi_version": (C.c_int, []),
    "icb_last_error": (C.c_char_p, []),
    "icb_device_count": (C.c_int, [_P(C.c_int)]),
    "icb_create": (C.c_int, [_P(Config), _P(_H)]),
    "icb_destroy": (C.c_int, [_H]),
    "icb_set_stream": (C.c_int, [_H, C.c_void_p]),
    "icb_synchronize": (C.c_int, [_H]),
    "icb_upload_ions": (C.c_int, [_H, C.c_uint64, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP, _U8P, _DP, _U64P, C.c_uint64]),
    "icb_download_ions": (C.c_int, [_H, _DP, _DP, _DP, _DP, _DP, _DP, _U8P, _DP, _DP]),
    "icb_update_state": (C.c_int, [_H, _DP, _DP, _DP, _DP, _DP, _DP, _U8P]),
    "icb_ion_count": (C.c_uint64, [_H]),
    "icb_advance": (C.c_int, [_H, C.c_uint64, _P(RunStats)]),
    "icb_advance_host": (C.c_int, [_H, C.c_uint64, C.c_int, _DP, _DP, _DP, _DP, _DP, _DP, _U8P, _P(RunStats)]),
    "icb_push": (C.c_int, [_H]),
    "icb_collide": (C.c_int, [_H, _P(RunStats)]),
    "icb_finalize": (C.c_int, [_H, _P(RunStats)]),
    "icb_get_clock": (C.c_int, [_H, _U64P, _DP]),
    "icb_set_clock": (C.c_int, [_H, C.c_uint64, _DP]),
    "icb_moments": (C.c_int, [_H, _DP]),
    "icb_mark_reference": (C.c_int, [_H]),
    "icb_autotune": (C.c_int, [_H, C.c_uint64, _P(Tuning)]),
    "icb_spacecharge_configure": (C.c_int, [_H, _P(SpaceChargeConfig)]),
    "icb_spacecharge_field": (C.c_int, [_H, _DP, _DP, _DP]),
    "icb_spacecharge_set_peers": (C.c_int, [_H, C.c_uint64, C.c_void_p, C.c_uint64, C.c_uint64]),
    "icb_spacecharge_export": (C.c_int, [_H, C.c_void_p]),
    "icb_ipm_deflection": (C.c_int, [C.c_int, _P(IpmPotential), C.c_uint64, _DP, _DP, _DP]),
    "icb_ipm_configure": (C.c_int, [_H, _P(IpmConfig)]),
    "icb_ipm_table": (C.c_int, [_H, _FP]),
    "icb_ipm_set_mlp": (C.c_int, [_H, _FP]),
    "icb_ehss_set_geometry": (C.c_int, [_H, C.c_int32, C.c_int32, _DP, _DP, C.c_double]),
    "icb_set_waveform": (C.c_int, [_H, C.c_int32, C.c_int32, _P(Waveform)]),
    "icb_set_tims_field": (C.c_int, [_H, C.c_int32, _P(TimsField)]),
    "icb_mlp_init": (C.c_int, [C.c_uint64, _FP]),
    "icb_mlp_train": (C.c_int, [C.c_int, _P(MlpTrainConfig), C.c_uint64, _FP, _FP, _FP, _DP]),
    "icb_mlp_forward": (C.c_int, [C.c_int, _FP, C.c_uint64, _FP, _FP, C.c_int]),
    "icb_mlp_gradients": (C.c_int, [C.c_int, _FP, C.c_uint64, _FP, _FP, _FP, _DP]),
    "icb_generate_ions": (C.c_int, [C.c_uint32, C.c_int32, _P(SpeciesSpec), _DP, _DP, _DP, _DP, _DP, _DP, _DP, _DP]),
    "icb_philox_eval": (C.c_int, [C.c_int, C.c_uint64, _U32P, C.c_uint64, C.c_int, _U32P]),
    "icb_clock_math_eval": (C.c_int, [C.c_int, C.c_uint64, _FP, C.c_int, _FP]),
    "icb_moments_noalloc": (C.c_int, [C.c_int, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m icarion_b200.build` "
                "(the package has no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != ICB_OK:
        msg = lib().icb_last_error().decode(errors="replace")
        raise IcbError(rc, msg)


def fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_FP)


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "expected contiguous float64"
    return a.ctypes.data_as(_DP)


def u8ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_U8P)


def u64ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_U64P)


def u32ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_U32P)
