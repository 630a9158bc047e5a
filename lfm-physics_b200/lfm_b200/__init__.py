"""lfm_b200: the lfm-physics leapfrog hot path, B200-native.

A drop-in for the reference's GPU path (lfm.Simulation -> Evolver ->
backend.step_*): the fused GOV-01 + GOV-02 step over the 19-point
Laplacian at the REAL, COMPLEX and COLOR levels and the S_a Helmholtz solve,
on hand-written sm_100a kernels in liblfm_b200.so (C ABI:
include/lfm_b200.h).  There is no CPU fallback.
"""

from .config import (
    BoundaryType,
    FieldLevel,
    SimulationConfig,
    full_physics,
    gravity_em,
    gravity_only,
)

__all__ = [
    "BoundaryType",
    "FieldLevel",
    "SimulationConfig",
    "full_physics",
    "gravity_em",
    "gravity_only",
    "B200Backend",
    "Evolver",
    "SplitChiEvolver",
    "get_backend",
]


def __getattr__(name):
    # The GPU-facing classes load the CUDA library on first use.
    if name in ("B200Backend", "get_backend"):
        from . import backend

        return getattr(backend, name)
    if name == "Evolver":
        from .evolver import Evolver

        return Evolver
    if name == "SplitChiEvolver":
        from .split import SplitChiEvolver

        return SplitChiEvolver
    raise AttributeError(name)
