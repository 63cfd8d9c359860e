"""B200-native active multi-phase-field cell update (Palmieri et al. 2015).

Python binding over the C ABI of ``libpfb200.so`` (``include/pfb200.h``). The
compute path is hand-written sm_100a CUDA; this package only marshals
arguments. There is no CPU fallback: importing works without a GPU, but every
device call needs the built library and a CUDA device.
"""
from ._abi import (CELL_DTYPE, CLASSES, FLAG_COUNT, FLAG_NAMES, LIB_PATH, TILE_AREA,
                   TILE_PITCH, TRAJ_DTYPE, Cell2D, Params2D, PfbError, StepArgs2D, TrajCell2D,
                   check, exported_symbols, lib, ptr)
from . import _abi3d  # registers the 3D entry points before the library loads
from . import _abi_sur  # registers the surrogate entry points
from ._abi3d import (CELL3D_DTYPE, FLAG3D_COUNT, FLAG3D_NAMES, Cell3D, Layout3D, MeasureArgs3D,
                     UpdateArgs3D)
from .sim2d import (Sim2D, SimParams2D, domain_side_for, fatal, flags_report,
                    grid_jitter_centres, palmieri_centres, step_coefficients, window_view,
                    world_field)
from .ensemble import Ensemble2D
from .surrogate import Surrogate2D
from . import checkpoint
from .sim3d import (Sim3D, SimParams3D, automatic_brick_edge, calibrate_seed_radius,
                    flags_report3, sequential_centres)

__all__ = [
    "CELL_DTYPE", "CLASSES", "FLAG_COUNT", "FLAG_NAMES", "LIB_PATH", "TILE_AREA", "TILE_PITCH",
    "TRAJ_DTYPE", "Cell2D", "Params2D", "PfbError", "StepArgs2D", "TrajCell2D", "check",
    "exported_symbols", "lib", "ptr", "Sim2D", "SimParams2D", "domain_side_for", "fatal",
    "flags_report", "grid_jitter_centres", "palmieri_centres", "step_coefficients",
    "window_view", "world_field", "CELL3D_DTYPE", "FLAG3D_COUNT", "FLAG3D_NAMES", "Cell3D",
    "Layout3D", "MeasureArgs3D", "UpdateArgs3D", "Sim3D", "SimParams3D", "automatic_brick_edge",
    "calibrate_seed_radius", "flags_report3", "sequential_centres", "Ensemble2D",
    "Surrogate2D",
]
