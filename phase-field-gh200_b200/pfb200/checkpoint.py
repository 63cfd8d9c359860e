"""The reference's 2D checkpoint file (PF "CELL" schema 1) over
``include/pfb200_ckpt.h``: read, write, and restart a Sim2D from a file
(reference src/checkpoint.cu:348-1011)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import CELL_DTYPE, TILE_AREA, Params2D, check, lib

P = C.c_void_p
I = C.c_int


class CkptParams2D(C.Structure):
    """The 192-byte parameter record (reference CheckpointParamsRecord)."""
    _pack_ = 1
    _fields_ = [
        ("Nx", C.c_int32), ("Ny", C.c_int32), ("dx", C.c_double), ("dy", C.c_double),
        ("dt", C.c_double), ("t_end", C.c_double), ("rho", C.c_double), ("lambda_", C.c_double),
        ("gamma_normal", C.c_double), ("gamma_soft", C.c_double), ("soft_fraction", C.c_double),
        ("kappa", C.c_double), ("target_radius", C.c_double), ("mu", C.c_double),
        ("v_A", C.c_double), ("v_A_sigma", C.c_double), ("xi", C.c_double), ("tau", C.c_double),
        ("seed", C.c_uint64), ("polarity_seed", C.c_uint64), ("initialization_hash", C.c_uint64),
        ("print_interval", C.c_int32), ("full_moment_every", C.c_int32),
        ("verify_every", C.c_int32), ("save_interval", C.c_int32),
        ("trajectory_samples", C.c_int32), ("reserved", C.c_int32),
        ("trajectory_interval", C.c_int64),
    ]


assert C.sizeof(CkptParams2D) == 192


class CkptInfo2D(C.Structure):
    _fields_ = [("step", C.c_longlong), ("time", C.c_double), ("num_cells", C.c_int),
                ("L", C.c_int), ("had_mobility", C.c_int)]


_abi._SIGS.update({
    "pfb_ckpt2d_params_from": (I, [C.POINTER(Params2D), C.POINTER(CkptParams2D)]),
    "pfb_ckpt2d_params_to": (I, [C.POINTER(CkptParams2D), I, C.POINTER(Params2D)]),
    "pfb_ckpt2d_read": (I, [C.c_char_p, C.POINTER(CkptInfo2D), C.POINTER(CkptParams2D), P, P]),
    "pfb_ckpt2d_write": (I, [C.c_char_p, C.POINTER(CkptParams2D), C.c_longlong, I, P, P]),
    "pfb_sim2d_write_checkpoint": (I, [P, C.c_char_p, C.POINTER(CkptParams2D)]),
    "pfb_sim2d_create_from_checkpoint": (P, [C.c_char_p, I]),
})


@dataclass
class Checkpoint2D:
    step: int
    time: float
    params: CkptParams2D
    cells: np.ndarray   # CELL_DTYPE records as a restart builds them
    phi: np.ndarray     # (N, 288, 288) float32 tiles
    had_mobility: bool


def _path(p) -> bytes:
    return str(p).encode()


def params_record(sim_params) -> CkptParams2D:
    """Record of a run with these SimParams2D (reference defaults elsewhere)."""
    rec = CkptParams2D()
    pc = sim_params.to_c()
    check(lib().pfb_ckpt2d_params_from(C.byref(pc), C.byref(rec)), "params_from")
    return rec


def read(path) -> Checkpoint2D:
    info, rec = CkptInfo2D(), CkptParams2D()
    check(lib().pfb_ckpt2d_read(_path(path), C.byref(info), C.byref(rec), None, None), "read")
    cells = np.zeros(info.num_cells, CELL_DTYPE)
    phi = np.zeros((info.num_cells, 288, 288), np.float32)
    check(lib().pfb_ckpt2d_read(_path(path), C.byref(info), C.byref(rec), cells.ctypes.data,
                                phi.ctypes.data), "read")
    return Checkpoint2D(info.step, info.time, rec, cells, phi, bool(info.had_mobility))


def write(path, rec: CkptParams2D, step: int, cells: np.ndarray, phi: np.ndarray) -> None:
    cells = np.ascontiguousarray(cells, CELL_DTYPE)
    phi = np.ascontiguousarray(phi, np.float32)
    assert phi.size == cells.size * TILE_AREA
    check(lib().pfb_ckpt2d_write(_path(path), C.byref(rec), step, cells.size, cells.ctypes.data,
                                 phi.ctypes.data), "write")


def write_sim(sim, path, rec: CkptParams2D | None = None) -> None:
    rec = rec if rec is not None else params_record(sim.params)
    check(lib().pfb_sim2d_write_checkpoint(sim._h, _path(path), C.byref(rec)), "write_checkpoint")


def restart(path, device: int = 0):
    """A Sim2D continuing from the checkpoint at `path`."""
    from .sim2d import Sim2D, SimParams2D
    ck = read(path)
    pc = Params2D()
    check(lib().pfb_ckpt2d_params_to(C.byref(ck.params), ck.cells.size, C.byref(pc)), "params_to")
    from dataclasses import fields
    p = SimParams2D(**{f.name: getattr(pc, f.name) for f in fields(SimParams2D)})
    return Sim2D(p, cells=ck.cells, phi=ck.phi, step=ck.step, device=device)
