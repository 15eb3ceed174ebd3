"""Interaction-potential collisions: the ion-neutral potential, its
deflection function (device quadrature), the cos(chi) table of a handle and
the learned deflection network (training, evaluation, loading).

Default potential: the reference's LJ1264 form (interaction_potential_
precompute.cpp:1386-1508) for an ion in N2 with a 12-6 well of 5 meV at
r_m = 4 A plus the induced-dipole term of the N2 polarisability 1.74 A^3
(utils/constants.h:54) for a singly charged ion; ion mass 300 Da.  The
collision event cross-section is pi b_max^2 with b_max = 12 A.  The network
is trained on centre-of-mass energies 1 meV - 10 eV (E_min_J .. E_max_J);
the table covers 0.01 meV - 10 eV (table_E_min_J .. E_max_J), so that the
slowest thermal encounters (about 0.6 % of collisions at 300 K fall below
1 meV) are deflected at their own energy, and serves the network outside
its range.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _capi as capi
from . import config as cfg
from . import sweep

EV_J = 1.602176634e-19


@dataclass
class IpmSetup:
    epsilon_J: float = 5e-3 * EV_J
    r_m_m: float = 4e-10
    polarizability_m3: float = 1.74e-30
    charge_C: float = cfg.ELEM_CHARGE_C
    b_max_m: float = 12e-10
    E_min_J: float = 1e-3 * EV_J          # trained range of the network
    E_max_J: float = 10.0 * EV_J
    table_E_min_J: float = 1e-5 * EV_J    # table range: table_E_min_J .. E_max_J
    n_E: int = 640
    n_b: int = 256

    def potential(self) -> capi.IpmPotential:
        p = capi.IpmPotential()
        p.epsilon_J = self.epsilon_J
        p.r_m_m = self.r_m_m
        p.polarizability_m3 = self.polarizability_m3
        p.charge_C = self.charge_C
        return p

    def config(self) -> capi.IpmConfig:
        c = capi.IpmConfig()
        c.potential = self.potential()
        c.b_max_m = self.b_max_m
        c.E_min_J = self.table_E_min_J
        c.E_max_J = self.E_max_J
        c.n_E = self.n_E
        c.n_b = self.n_b
        c.net_E_min_J = self.E_min_J
        c.net_E_max_J = self.E_max_J
        return c

    def table_grid(self) -> tuple[np.ndarray, np.ndarray]:
        """(E [n_E], b [n_b]) nodes of the handle's cos(chi) table."""
        lnE = np.linspace(math.log(self.table_E_min_J), math.log(self.E_max_J), self.n_E)
        return np.exp(lnE), np.linspace(0.0, self.b_max_m, self.n_b)

    def table_scale(self) -> tuple[float, float]:
        """(ln E_min, (n_E - 1) / ln(E_max / E_min)) of the table."""
        lo = math.log(self.table_E_min_J)
        return lo, (self.n_E - 1) / (math.log(self.E_max_J) - lo)

    def coefficients(self) -> tuple[float, float, float]:
        """(c12, c6, c4) of V = c12/r^12 - c6/r^6 - c4/r^4."""
        sigma = self.r_m_m * 2.0 ** (-1.0 / 6.0)
        c12 = 4.0 * self.epsilon_J * sigma ** 12
        c6 = 4.0 * self.epsilon_J * sigma ** 6
        c4 = 0.5 * self.polarizability_m3 * 8.987551787e9 * self.charge_C ** 2
        return c12, c6, c4


def deflection(setup: IpmSetup, E_J: np.ndarray, b_m: np.ndarray, device: int = 0) -> np.ndarray:
    """cos(chi) of the device quadrature."""
    E = np.ascontiguousarray(E_J, dtype=np.float64)
    b = np.ascontiguousarray(b_m, dtype=np.float64)
    out = np.zeros_like(E)
    pot = setup.potential()
    capi.check(capi.lib().icb_ipm_deflection(device, C.byref(pot), E.size, capi.dptr(E), capi.dptr(b),
                                             capi.dptr(out)))
    return out


def normalize(setup: IpmSetup, E_J: np.ndarray, b_m: np.ndarray) -> np.ndarray:
    """Network inputs (2n float32): 2 (ln E - ln E_min)/(ln E_max - ln E_min) - 1, 2 b/b_max - 1."""
    lo, hi = math.log(setup.E_min_J), math.log(setup.E_max_J)
    x0 = 2.0 * (np.log(E_J) - lo) / (hi - lo) - 1.0
    x1 = 2.0 * np.asarray(b_m) / setup.b_max_m - 1.0
    return np.ascontiguousarray(np.stack([x0, x1], axis=1).ravel(), dtype=np.float32)


def training_set(setup: IpmSetup, n: int = 2 ** 20, seed: int = 2024, device: int = 0):
    """n (E, b) pairs, E log-uniform over [E_min, E_max], b uniform over
    [0, b_max], with cos(chi) from the quadrature: (x, y, E, b)."""
    rng = np.random.default_rng(seed)
    E = np.exp(rng.uniform(math.log(setup.E_min_J), math.log(setup.E_max_J), n))
    b = rng.uniform(0.0, setup.b_max_m, n)
    y = deflection(setup, E, b, device).astype(np.float32)
    return normalize(setup, E, b), y, E, b


def init_params(seed: int = 7) -> np.ndarray:
    p = np.zeros(capi.MLP_N_PARAMS, dtype=np.float32)
    capi.check(capi.lib().icb_mlp_init(seed, capi.fptr(p)))
    return p


def train(x: np.ndarray, y: np.ndarray, params: np.ndarray | None = None, epochs: int = 30, batch: int = 1024,
          lr: float = 3e-3, lr_min: float = 1e-5, seed: int = 7, bf16_forward: bool = True,
          device: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Adam on the device; returns (params, loss per epoch)."""
    p = init_params(seed) if params is None else np.array(params, dtype=np.float32, copy=True)
    c = capi.MlpTrainConfig()
    c.epochs = epochs
    c.batch = batch
    c.lr = lr
    c.lr_min = lr_min
    c.seed = seed
    c.bf16_forward = int(bf16_forward)
    losses = np.zeros(epochs)
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    capi.check(capi.lib().icb_mlp_train(device, C.byref(c), y.size, capi.fptr(x), capi.fptr(y), capi.fptr(p),
                                        capi.dptr(losses)))
    return p, losses


def forward(params: np.ndarray, x: np.ndarray, mode: int = 1, device: int = 0) -> np.ndarray:
    """mode 0: FP32 arithmetic; mode 1: the collision path's BF16 tensor-core evaluation."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.zeros(x.size // 2, dtype=np.float32)
    capi.check(capi.lib().icb_mlp_forward(device, capi.fptr(np.ascontiguousarray(params, dtype=np.float32)),
                                          y.size, capi.fptr(x), capi.fptr(y), mode))
    return y


def gradients(params: np.ndarray, x: np.ndarray, y: np.ndarray, device: int = 0) -> tuple[np.ndarray, float]:
    g = np.zeros(capi.MLP_N_PARAMS, dtype=np.float32)
    loss = C.c_double(0.0)
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    capi.check(capi.lib().icb_mlp_gradients(device, capi.fptr(np.ascontiguousarray(params, dtype=np.float32)),
                                            y.size, capi.fptr(x), capi.fptr(y), capi.fptr(g), C.byref(loss)))
    return g, loss.value


def drift_ensembles(setup: IpmSetup, en_td=(10.0, 40.0, 80.0), n_total: int = 1 << 20, ion_mass_amu: float = 300.0,
                    seed: int = 123):
    """The learned-IPM evaluation workload: n_total ions of ion_mass_amu, +1,
    split evenly over one IMS drift ensemble per E/N (N2, 300 K, 1000 Pa,
    event radius b_max, dt = 0.1 / nu_max at that E/N).  Returns
    (ensembles, initial IonState, ensemble offsets)."""
    from .sim import generate_ions
    counts = [n_total // len(en_td) + (1 if k < n_total % len(en_td) else 0) for k in range(len(en_td))]
    m_ion = ion_mass_amu * cfg.AMU_TO_KG
    sigma_ev = math.pi * setup.b_max_m ** 2
    ensembles, specs = [], []
    for e_td, c in zip(en_td, counts):
        nu = sweep.collision_frequency_max(e_td, m_ion, sigma_ev, cfg.GAS_MASS_KG["N2"], 300.0, 1000.0)
        domain = {"instrument": "IMS", "geometry": {"origin_m": [0.0, 0.0, -0.01], "length_m": 0.1, "radius_m": 0.05},
                  "env": {"temperature_K": 300.0, "pressure_Pa": 1000.0, "gas_species": "N2"},
                  "fields": {"DC": {"EN_Td": e_td}}}
        ensembles.append(cfg.ensemble_params(domain, 0.0, 0.1 / nu, ipm_bmax_m=setup.b_max_m))
        specs.append(cfg.species_spec(c, m_ion, cfg.ELEM_CHARGE_C,
                                      {"type": "gaussian", "center": [0, 0, 0], "std": [5e-4] * 3},
                                      {"type": "thermal", "temperature_K": 300.0}))
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    return ensembles, generate_ions(seed, specs), offsets
