"""icarion_b200 — B200-native uniform-dt batch step of the ICARION ion
trajectory simulator (Boris/RK4 push through analytic fields fused with
stochastic buffer-gas collisions), behind the reference's plug points.

The compute path is the in-tree CUDA library ``_lib/libicarion_b200.so``
(sm_100a); there is no CPU fallback.
"""
from . import _capi as capi
from .sim import IonState, Simulation, device_count, generate_ions

__all__ = ["capi", "IonState", "Simulation", "generate_ions", "device_count"]
