"""ctypes mirror of ``include/pfb200.h`` and the library loader.

The records are byte-for-byte the reference's ``pf::CellState`` (192 B) and
``pf::StepArgs`` (216 B) (reference include/kernels.cuh:27-57, :74-116). The
loader never falls back to anything: if ``libpfb200.so`` is missing or fails to
load, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libpfb200.so"

FLAG_NAMES = (
    "S_overflow",
    "q_clamp",
    "support_clip",
    "class_exhausted",
    "S_other_negative",
    "phi_nonfinite",
    "V_nonpositive",
    "class_unsupported",
)
FLAG_COUNT = 8
FATAL_FLAGS = tuple(i for i in range(FLAG_COUNT) if i != 2)
TILE_PITCH = 288
TILE_AREA = 288 * 288
# (wx, wy, tx0, ty0) of the six shape classes (reference include/params.cuh:138-147)
CLASSES = ((144, 144, 64, 64), (176, 144, 32, 64), (144, 176, 64, 32),
           (160, 160, 32, 32), (224, 224, 32, 32), (286, 286, 1, 1))


class AdvectionAccum(C.Structure):
    _fields_ = [("q", C.c_double * 6), ("count", C.c_ulonglong)]


class Cell2D(C.Structure):
    _fields_ = [
        ("gx0", C.c_int32), ("gy0", C.c_int32),
        ("cls", C.c_uint8), ("cls_written", C.c_uint8 * 2), ("pad0", C.c_uint8),
        ("global_id", C.c_int32),
        ("gamma", C.c_float), ("v_A", C.c_float), ("R_tgt", C.c_float),
        ("theta", C.c_float),
        ("V", C.c_double), ("Cx", C.c_double), ("Cy", C.c_double), ("perim", C.c_double),
        ("bb_lo_x", C.c_int32), ("bb_hi_x", C.c_int32),
        ("bb_lo_y", C.c_int32), ("bb_hi_y", C.c_int32),
        ("vx", C.c_float), ("vy", C.c_float),
        ("Ix", C.c_double), ("Iy", C.c_double),
        ("promote_ctr", C.c_uint32), ("shift_ctr", C.c_uint32), ("tumble_ctr", C.c_uint32),
        ("phi_max", C.c_float),
        ("reserved", C.c_uint32 * 2),
        ("advection", AdvectionAccum),
        ("reserved_unused", C.c_uint32),
        ("M_pf", C.c_float),
        ("_tail", C.c_uint8 * 0),
    ]


assert C.sizeof(Cell2D) == 192, C.sizeof(Cell2D)

CELL_DTYPE = np.dtype({
    "names": ["gx0", "gy0", "cls", "cls_written", "pad0", "global_id", "gamma", "v_A",
              "R_tgt", "theta", "V", "Cx", "Cy", "perim", "bb_lo_x", "bb_hi_x", "bb_lo_y",
              "bb_hi_y", "vx", "vy", "Ix", "Iy", "promote_ctr", "shift_ctr", "tumble_ctr",
              "phi_max", "reserved", "adv_q", "adv_count", "reserved_unused", "M_pf"],
    "formats": ["<i4", "<i4", "u1", ("u1", 2), "u1", "<i4", "<f4", "<f4", "<f4", "<f4",
                "<f8", "<f8", "<f8", "<f8", "<i4", "<i4", "<i4", "<i4", "<f4", "<f4",
                "<f8", "<f8", "<u4", "<u4", "<u4", "<f4", ("<u4", 2), ("<f8", 6), "<u8",
                "<u4", "<f4"],
    "offsets": [0, 4, 8, 9, 11, 12, 16, 20, 24, 28, 32, 40, 48, 56, 64, 68, 72, 76, 80, 84,
                88, 96, 104, 108, 112, 116, 120, 128, 176, 184, 188],
    "itemsize": 192,
})


class StepArgs2D(C.Structure):
    _fields_ = [
        ("phi_in", C.c_void_p), ("phi_out", C.c_void_p),
        ("S_rd", C.c_void_p), ("S_sc", C.c_void_p), ("S_cl", C.c_void_p),
        ("cell", C.c_void_p), ("cell_cls", C.c_void_p), ("perm", C.c_void_p),
        ("cursor_use", C.c_void_p), ("cursor_clear", C.c_void_p),
        ("step_rd", C.c_void_p), ("step_wr", C.c_void_p),
        ("flags", C.c_void_p), ("moments", C.c_void_p),
        ("physical_dt", C.c_double),
        ("N", C.c_int), ("L", C.c_int), ("P", C.c_int), ("parity_out", C.c_int),
        ("dt", C.c_float),
        ("A0", C.c_double), ("vol_scale", C.c_double),
        ("bulk_scale", C.c_float), ("rep_coeff", C.c_float), ("mot_coeff", C.c_float),
        ("seed", C.c_ulonglong), ("polarity_seed", C.c_ulonglong),
        ("p_tumble", C.c_double),
        ("full_moment_every", C.c_int),
        ("clear_ahead_words", C.c_ulonglong),
    ]


assert C.sizeof(StepArgs2D) == 216, C.sizeof(StepArgs2D)


class Params2D(C.Structure):
    _fields_ = [
        ("L", C.c_int), ("num_cells", C.c_int),
        ("dt", C.c_double), ("lambda_", C.c_double), ("target_radius", C.c_double),
        ("kappa", C.c_double), ("mu", C.c_double), ("xi", C.c_double), ("tau", C.c_double),
        ("v_A", C.c_double), ("gamma_normal", C.c_double), ("gamma_cancer", C.c_double),
        ("cancer_fraction", C.c_double), ("v_A_sigma", C.c_double),
        ("phase_field_mobility", C.c_double),
        ("seed", C.c_ulonglong), ("polarity_seed", C.c_ulonglong),
        ("full_moment_every", C.c_int), ("phi_storage", C.c_int),
    ]


class TrajCell2D(C.Structure):
    _fields_ = [("global_id", C.c_int32), ("cls", C.c_int32), ("cx", C.c_float),
                ("cy", C.c_float), ("vx", C.c_float), ("vy", C.c_float),
                ("theta", C.c_float), ("volume", C.c_float), ("perim", C.c_float),
                ("gamma", C.c_float), ("v_A", C.c_float), ("phi_max", C.c_float)]


TRAJ_DTYPE = np.dtype([("global_id", "<i4"), ("cls", "<i4"), ("cx", "<f4"), ("cy", "<f4"),
                       ("vx", "<f4"), ("vy", "<f4"), ("theta", "<f4"), ("volume", "<f4"),
                       ("perim", "<f4"), ("gamma", "<f4"), ("v_A", "<f4"),
                       ("phi_max", "<f4")])

P = C.c_void_p
I = C.c_int
_SIGS = {
    "pfb_version": (C.c_char_p, []),
    "pfb_last_error": (C.c_char_p, []),
    "pfb_sizeof": (C.c_size_t, [I]),
    "pfb_step2d_configure": (I, []),
    "pfb_step2d_grid": (I, [I, I]),
    "pfb_step2d_launch": (I, [C.POINTER(StepArgs2D), I, P]),
    "pfb_step2d_launch_ex": (I, [C.POINTER(StepArgs2D), I, I, P]),
    "pfb_device_status": (I, [C.POINTER(C.c_uint), I]),
    "pfb_init_tiles2d": (I, [P, P, P, P, I, I, P, P, C.c_float, C.c_float, P]),
    "pfb_init_moments2d": (I, [P, P, P, I, P]),
    "pfb_scatter_all2d": (I, [P, P, P, P, I, I, I, P, P]),
    "pfb_zero_u32": (I, [P, C.c_size_t, P]),
    "pfb_verify_cells2d": (I, [P, P, P, I, P, P, P]),
    "pfb_verify_S": (I, [P, C.c_size_t, P, P]),
    "pfb_pack_traj2d": (I, [P, P, P, I, I, P]),
    "pfb_philox4x32_10": (None, [C.c_uint32] * 6 + [C.POINTER(C.c_uint32)]),
    "pfb_philox_uniform53": (C.c_double, [C.c_uint32, C.c_uint32]),
    "pfb_q_of": (C.c_uint32, [C.c_float]),
    "pfb_palmieri_centres": (I, [I, C.c_double, C.c_double, C.c_ulonglong, P, P]),
    "pfb_grid_jitter_centres": (I, [I, I, C.c_ulonglong, P, P]),
    "pfb_ic_theta": (C.c_float, [C.c_int32, C.c_ulonglong]),
    "pfb_ic_v_A": (C.c_double, [C.c_int32, C.c_ulonglong, C.c_double, C.c_double]),
    "pfb_domain_side_for": (I, [I, C.c_double, C.c_double]),
    "pfb_fill_coefficients2d": (I, [C.POINTER(Params2D), C.POINTER(StepArgs2D)]),
    "pfb_sim2d_create": (P, [C.POINTER(Params2D), P, P, I]),
    "pfb_sim2d_create_from_state": (P, [C.POINTER(Params2D), P, P, C.c_longlong, I]),
    "pfb_sim2d_destroy": (None, [P]),
    "pfb_sim2d_set_cluster": (I, [P, I]),
    "pfb_sim2d_set_graph": (I, [P, I]),
    "pfb_sim2d_set_variant": (I, [P, I]),
    "pfb_sim2d_scatter_recounts": (I, [P, C.POINTER(C.c_uint)]),
    "pfb_sim2d_set_visit_order": (I, [P, I]),
    "pfb_sim2d_visit_order": (I, [P, P]),
    "pfb_sim2d_advance": (I, [P, C.c_longlong]),
    "pfb_sim2d_sync": (I, [P]),
    "pfb_sim2d_step": (C.c_longlong, [P]),
    "pfb_sim2d_side": (I, [P]),
    "pfb_sim2d_pitch": (I, [P]),
    "pfb_sim2d_num_cells": (I, [P]),
    "pfb_sim2d_get_cells": (I, [P, P]),
    "pfb_sim2d_get_phi": (I, [P, P]),
    "pfb_sim2d_get_S": (I, [P, P]),
    "pfb_sim2d_get_flags": (I, [P, P]),
    "pfb_sim2d_set_state": (I, [P, P, P, C.c_longlong]),
    "pfb_sim2d_pack_traj": (I, [P, P]),
    "pfb_sim2d_advance_record": (I, [P, C.c_longlong, I, P, I]),
    "pfb_ens2d_advance_record": (I, [P, C.c_longlong, I, P, I]),
    "pfb_ens2d_stream": (P, [P]),
    "pfb_sim2d_save": (I, [P]),
    "pfb_sim2d_restore": (I, [P]),
    "pfb_sim2d_velocity_open": (I, [P, C.c_char_p, I, C.c_longlong, I]),
    "pfb_sim2d_velocity_capture": (I, [P]),
    "pfb_sim2d_velocity_last_frame": (C.c_longlong, [P]),
    "pfb_sim2d_velocity_close": (I, [P]),
    "pfb_sim2d_verify": (I, [P, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_uint32)]),
    "pfb_sim2d_boundary_open": (I, [P, C.c_char_p, C.c_longlong, I]),
    "pfb_sim2d_boundary_capture": (I, [P]),
    "pfb_sim2d_boundary_close": (I, [P]),
    "pfb_step2d_launch_observed": (I, [C.POINTER(StepArgs2D), I, I, P]),
    "pfb_velocity_moments2d": (I, [C.POINTER(StepArgs2D), P, C.c_double, P]),
    "pfb_sim2d_bench": (I, [P, I, I, C.POINTER(C.c_double)]),
    "pfb_sim2d_step_args": (I, [P, C.POINTER(StepArgs2D)]),
    "pfb_sim2d_stream": (P, [P]),
    "pfb_ens2d_create": (P, [I, C.POINTER(Params2D), P, P, I]),
    "pfb_ens2d_destroy": (None, [P]),
    "pfb_ens2d_num_systems": (I, [P]),
    "pfb_ens2d_set_cluster": (I, [P, I]),
    "pfb_ens2d_autotune": (I, [P, I, C.POINTER(C.c_int)]),
    "pfb_ens2d_advance": (I, [P, I]),
    "pfb_ens2d_advance_serial": (I, [P, I]),
    "pfb_ens2d_sync": (I, [P]),
    "pfb_ens2d_step": (C.c_longlong, [P]),
    "pfb_ens2d_system": (P, [P, I]),
    "pfb_ens2d_bench": (I, [P, I, I, I, C.POINTER(C.c_double)]),
}

_LIB = None


class PfbError(RuntimeError):
    """A C-ABI call returned a negative status."""


def lib() -> C.CDLL:
    """Load ``libpfb200.so`` (built by ``build.py``; ``PFB_LIB`` names another
    build of it); raise if it is absent."""
    global _LIB
    if _LIB is None:
        path = Path(os.environ.get("PFB_LIB") or LIB_PATH)
        if not path.exists():
            raise RuntimeError(
                f"{path} is missing: build it with "
                "`python phase-field-gh200_b200/build.py` (there is no fallback path)")
        L = C.CDLL(str(path))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(rc: int, what: str = "") -> int:
    if rc is not None and rc < 0:
        msg = lib().pfb_last_error().decode(errors="replace")
        raise PfbError(f"{what}: status {rc}: {msg}")
    return rc


def ptr(a) -> int | None:
    """Address of a numpy array's data (or a torch tensor's), None for None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return int(a)
