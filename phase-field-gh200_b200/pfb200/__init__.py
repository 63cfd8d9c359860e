"""B200-native active multi-phase-field cell update (Palmieri et al. 2015).

Python binding over the C ABI of ``libpfb200.so`` (``include/pfb200.h``). The
compute path is hand-written sm_100a CUDA; this package only marshals
arguments. There is no CPU fallback: importing works without a GPU, but every
device call needs the built library and a CUDA device.
"""
from ._abi import (CELL_DTYPE, CLASSES, FLAG_COUNT, FLAG_NAMES, LIB_PATH, TILE_AREA,
                   TILE_PITCH, TRAJ_DTYPE, Cell2D, Params2D, PfbError, StepArgs2D, TrajCell2D,
                   check, exported_symbols, lib, ptr)
from .sim2d import (Sim2D, SimParams2D, domain_side_for, fatal, flags_report,
                    grid_jitter_centres, palmieri_centres, step_coefficients, window_view,
                    world_field)

__all__ = [
    "CELL_DTYPE", "CLASSES", "FLAG_COUNT", "FLAG_NAMES", "LIB_PATH", "TILE_AREA", "TILE_PITCH",
    "TRAJ_DTYPE", "Cell2D", "Params2D", "PfbError", "StepArgs2D", "TrajCell2D", "check",
    "exported_symbols", "lib", "ptr", "Sim2D", "SimParams2D", "domain_side_for", "fatal",
    "flags_report", "grid_jitter_centres", "palmieri_centres", "step_coefficients",
    "window_view", "world_field",
]
