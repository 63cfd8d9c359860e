"""The reference's checkpoint files over ``include/pfb200_ckpt.h``: the 2D
PF "CELL" schema 1 (reference src/checkpoint.cu:348-1011) and the 3D PF3D
schema 1 (reference src/pf3d/checkpoint.cu:116-1235): read, write, and
restart a Sim2D / Sim3D from a file."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import CELL_DTYPE, TILE_AREA, Params2D, check, lib
from ._abi3d import CELL3D_DTYPE, Params3D

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


class CkptParams3D(C.Structure):
    """The 288-byte PF3D parameter record (reference ParamsRecord3D)."""
    _pack_ = 1
    _fields_ = [
        ("Nx", C.c_int64), ("Ny", C.c_int64), ("Nz", C.c_int64),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("brick_edge", C.c_uint32), ("boundary_flags", C.c_uint32),
        ("dt", C.c_double), ("t_end", C.c_double), ("lambda_", C.c_double),
        ("gamma_normal", C.c_double), ("gamma_soft", C.c_double), ("soft_fraction", C.c_double),
        ("kappa", C.c_double), ("target_radius", C.c_double), ("mu", C.c_double),
        ("v_A", C.c_double), ("v_A_sigma", C.c_double), ("xi", C.c_double), ("tau", C.c_double),
        ("volume_fraction", C.c_double), ("seed", C.c_uint64), ("polarity_seed", C.c_uint64),
        ("print_interval", C.c_int64), ("full_moment_every", C.c_int64),
        ("verify_every", C.c_int64), ("integrator_id", C.c_uint32), ("stencil_id", C.c_uint32),
        ("rng_id", C.c_uint32), ("trajectory_interval", C.c_uint32),
        ("initialization_hash", C.c_uint64), ("aging_time", C.c_double),
        ("promoted_measure_policy", C.c_uint64), ("promoted_measure_auto_wave_ctas", C.c_uint64),
        ("channel_height", C.c_int64), ("channel_padding", C.c_int64),
        ("wall_kappa", C.c_double), ("wall_width", C.c_double),
    ]


assert C.sizeof(CkptParams3D) == 288


class CkptInfo3D(C.Structure):
    _fields_ = [("step", C.c_longlong), ("time", C.c_double), ("num_cells", C.c_int),
                ("brick_edge", C.c_int), ("base_measure_shards", C.c_int), ("crc64", C.c_uint64)]


_abi._SIGS.update({
    "pfb_crc64_ecma": (C.c_uint64, [C.c_uint64, C.c_char_p, C.c_size_t]),
    "pfb_ckpt3d_params_from": (I, [C.POINTER(Params3D), I, C.POINTER(CkptParams3D)]),
    "pfb_ckpt3d_params_to": (I, [C.POINTER(CkptParams3D), I, C.POINTER(Params3D)]),
    "pfb_ckpt3d_read": (I, [C.c_char_p, C.POINTER(CkptInfo3D), C.POINTER(CkptParams3D), P, P]),
    "pfb_ckpt3d_payload_words": (I, [C.c_char_p, C.POINTER(C.c_ulonglong)]),
    "pfb_ckpt3d_write": (I, [C.c_char_p, C.POINTER(CkptParams3D), C.c_longlong, I, P, P, I]),
    "pfb_sim3d_write_checkpoint": (I, [P, C.c_char_p, C.POINTER(CkptParams3D)]),
    "pfb_sim3d_create_from_checkpoint_ex": (P, [C.c_char_p, I, I, I]),
    "pfb_sim3d_create_from_checkpoint": (P, [C.c_char_p, I]),
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


# ---- 3D -------------------------------------------------------------------------

@dataclass
class Checkpoint3D:
    step: int
    time: float
    params: CkptParams3D
    cells: np.ndarray   # CELL3D_DTYPE records (storage_edge 0: base brick)
    packed: np.ndarray  # each cell's field in cell order, B^3 or E^3 values, x fastest
    brick_edge: int
    base_measure_shards: int
    crc64: int

    def edges(self) -> np.ndarray:
        """Cube edge of every cell (B for a base cell)."""
        e = self.cells["storage_edge"].astype(np.int64)
        return np.where(e > self.brick_edge, e, self.brick_edge)

    def fields(self) -> list[np.ndarray]:
        """Each cell's field as an (E, E, E) view (z, y, x)."""
        out, off = [], 0
        for e in self.edges():
            n = int(e) ** 3
            out.append(self.packed[off:off + n].reshape(int(e), int(e), int(e)))
            off += n
        return out

    @property
    def phi(self) -> np.ndarray:
        """(N, B, B, B) fields; only when no cell is on a promoted cube."""
        B = self.brick_edge
        if (self.edges() != B).any():
            raise ValueError("cells on promoted cubes: use fields() or packed")
        return self.packed.reshape(self.cells.size, B, B, B)


def params_record3d(sim_params, brick: int = 0) -> CkptParams3D:
    rec = CkptParams3D()
    pc = sim_params.to_c()
    check(lib().pfb_ckpt3d_params_from(C.byref(pc), brick, C.byref(rec)), "params_from")
    return rec


def read3d(path) -> Checkpoint3D:
    info, rec = CkptInfo3D(), CkptParams3D()
    words = C.c_ulonglong(0)
    check(lib().pfb_ckpt3d_payload_words(_path(path), C.byref(words)), "read")
    check(lib().pfb_ckpt3d_read(_path(path), C.byref(info), C.byref(rec), None, None), "read")
    cells = np.zeros(info.num_cells, CELL3D_DTYPE)
    packed = np.zeros(words.value, np.float32)
    check(lib().pfb_ckpt3d_read(_path(path), C.byref(info), C.byref(rec), cells.ctypes.data,
                                packed.ctypes.data), "read")
    return Checkpoint3D(info.step, info.time, rec, cells, packed, info.brick_edge,
                        info.base_measure_shards, info.crc64)


def write3d(path, rec: CkptParams3D, step: int, cells: np.ndarray, phi: np.ndarray,
            base_measure_shards: int = 4) -> None:
    cells = np.ascontiguousarray(cells, CELL3D_DTYPE)
    phi = np.ascontiguousarray(phi, np.float32)
    check(lib().pfb_ckpt3d_write(_path(path), C.byref(rec), step, cells.size, cells.ctypes.data,
                                 phi.ctypes.data, base_measure_shards), "write")


def write_sim3d(sim, path, rec: CkptParams3D | None = None) -> None:
    rec = rec if rec is not None else params_record3d(sim.params, sim.B)
    check(lib().pfb_sim3d_write_checkpoint(sim._h, _path(path), C.byref(rec)), "write_checkpoint")


def restart3d(path, device: int = 0, memory_mode: str = "auto", scratch_slots: int = 0):
    """A Sim3D continuing from the PF3D checkpoint at `path` (storage mode
    as Sim3D's)."""
    from .sim3d import GEOMETRIES, Sim3D, SimParams3D
    ck3 = read3d(path)
    pc = Params3D()
    check(lib().pfb_ckpt3d_params_to(C.byref(ck3.params), ck3.cells.size, C.byref(pc)), "params_to")
    geometry = {v: k for k, v in GEOMETRIES.items()}[pc.boundary_flags]
    from dataclasses import fields
    kw = {f.name: getattr(pc, f.name) for f in fields(SimParams3D) if f.name != "geometry"}
    p = SimParams3D(geometry=geometry, **kw)
    return Sim3D(p, cells=ck3.cells, phi=ck3.packed, step=ck3.step, device=device,
                 memory_mode=memory_mode, scratch_slots=scratch_slots)
