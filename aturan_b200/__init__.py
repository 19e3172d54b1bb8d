"""aturan_b200: B200 (sm_100a) kernels for ATURAN's dynamical-core time step.

The hot path of the reference (planet/RHS_Uran_Turb.cpp, RungeKutta_Uran_Turb.cpp,
PressureSolverUran.h, PressureSolver.h, SaturationAdjustment.h) as hand-written CUDA behind the
C ABI of include/aturan_b200.h. `Context` (aturan_b200.api) is the Python face of that ABI.
"""
from . import fields, params, state  # noqa: F401
from .params import Params, default_params, FP64, MIXED  # noqa: F401
