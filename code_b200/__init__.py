"""B200-native implementation of GETM's per-timestep 3D hot path (getm-model/code).

Public surface: :class:`code_b200.getm.Context` (the reference-named routines over the CUDA
library's C ABI), :class:`code_b200.grid.Grid` and the seeded synthetic cases in
:mod:`code_b200.cases`.
"""
from .grid import Grid, HALO  # noqa: F401

__all__ = ["Grid", "HALO"]
