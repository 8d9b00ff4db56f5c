"""B200 (sm_100a) implementation of MIMICA's dynamical-core hot path.

Flux-form scalar advection (WENO3-switch / PPM / MUSCL), FD4 momentum advection,
the Heun stage update and the anelastic pressure projection, as hand-written
CUDA kernels behind the C ABI of ``include/mimica_gpu.h``.
"""
from . import _lib
from .config import Domain, State, cumulus_domain, cumulus_state, warm_bubble_domain, warm_bubble_state
from .model import Mimica

__all__ = ["Domain", "State", "Mimica", "warm_bubble_domain", "warm_bubble_state", "cumulus_domain",
           "cumulus_state", "_lib"]
