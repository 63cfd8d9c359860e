"""ctypes mirror of ``include/pfb200_3d.h``.

The records are byte-for-byte the reference's ``pf3d::CellState3D`` (256 B),
``SLayout3D``, ``MeasureArgs3D`` (168 B), ``UpdateArgs3D`` (208 B),
``InitArgs3D`` and ``ScatterArgs3D`` (reference include/pf3d/kernels.cuh:
98-316). Importing this module registers the 3D entry points with the loader
in :mod:`._abi`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi

BOUNDARY_PERIODIC_XYZ = 0x7
BOUNDARY_SUBSTRATE_SLAB = 0x3
BOUNDARY_HARD_WALL_CHANNEL = 0xB
FLAG3D_NAMES = ("S_overflow", "q_clamp", "S_negative", "nonfinite", "V_nonpositive",
                "support_exhausted", "support_edge", "destination_clip", "invalid_geometry",
                "slab_top_contact")
FLAG3D_COUNT = 10
FATAL3D_MASK = 0x3BF


class Cell3D(C.Structure):
    _fields_ = [
        ("global_id", C.c_int64),
        ("origin_x", C.c_int64), ("origin_y", C.c_int64), ("origin_z", C.c_int64),
        ("polarity_x", C.c_float), ("polarity_y", C.c_float), ("polarity_z", C.c_float),
        ("velocity_x", C.c_float), ("velocity_y", C.c_float), ("velocity_z", C.c_float),
        ("gamma", C.c_float), ("v_A", C.c_float), ("R_tgt", C.c_float), ("phi_max", C.c_float),
        ("shift_ctr", C.c_uint32), ("tumble_ctr", C.c_uint32), ("flags", C.c_uint32),
        ("pad0", C.c_uint32),
        ("bb_lo_x", C.c_int32), ("bb_hi_x", C.c_int32), ("bb_lo_y", C.c_int32),
        ("bb_hi_y", C.c_int32), ("bb_lo_z", C.c_int32), ("bb_hi_z", C.c_int32),
        ("pending_shift_x", C.c_int32), ("pending_shift_y", C.c_int32),
        ("pending_shift_z", C.c_int32), ("pad1", C.c_uint32),
        ("V", C.c_double), ("Cx", C.c_double), ("Cy", C.c_double), ("Cz", C.c_double),
        ("surface", C.c_double), ("Ix", C.c_double), ("Iy", C.c_double), ("Iz", C.c_double),
        ("storage_edge", C.c_uint32), ("pad2", C.c_uint32),
        ("wall_overlap", C.c_double), ("outside_slit_volume", C.c_double),
        ("reserved", C.c_uint32 * 10),
        ("_pad_tail", C.c_uint8 * 0),
    ]


# numpy view of the same record (explicit offsets, 256-byte items)
_NP = {C.c_int64: "<i8", C.c_float: "<f4", C.c_uint32: "<u4", C.c_int32: "<i4",
       C.c_double: "<f8"}
_F = [(f, t) for f, t in Cell3D._fields_ if not f.startswith("_")]
CELL3D_DTYPE = np.dtype({
    "names": [f for f, _ in _F],
    "formats": [("<u4", (t._length_,)) if hasattr(t, "_length_") else _NP[t] for _, t in _F],
    "offsets": [getattr(Cell3D, f).offset for f, _ in _F],
    "itemsize": 256,
})


class Layout3D(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("pitch_x", C.c_int),
                ("boundary_flags", C.c_uint32)]


class Wall3D(C.Structure):
    _fields_ = [("values", C.c_void_p), ("planes", C.c_int)]


class Selection3D(C.Structure):
    _fields_ = [("ids", C.c_void_p), ("count", C.c_int)]


class Storage3D(C.Structure):
    _fields_ = [("z_cap", C.c_int)]


class MeasureArgs3D(C.Structure):
    _fields_ = [
        ("phi", C.c_void_p), ("S", C.c_void_p), ("wall", Wall3D), ("cells", C.c_void_p),
        ("global_flags", C.c_void_p), ("step", C.c_void_p), ("layout", Layout3D),
        ("N", C.c_int), ("B", C.c_int), ("partials", C.c_void_p), ("shards", C.c_int),
        ("polarity_stream", C.c_uint64), ("aging_steps", C.c_uint64), ("p_tumble", C.c_double),
        ("motility_coeff", C.c_float), ("max_shift", C.c_int), ("support_margin", C.c_int),
        ("apply_tumble", C.c_uint8), ("compute_surface", C.c_uint8),
        ("selection", Selection3D), ("storage", Storage3D),
    ]


class ExchangeRegion3D(C.Structure):
    _fields_ = [("y_lo", C.c_int * 4), ("y_hi", C.c_int * 4), ("y_count", C.c_int),
                ("z_lo", C.c_int), ("z_hi", C.c_int)]


class UpdateArgs3D(C.Structure):
    _fields_ = [
        ("phi_in", C.c_void_p), ("phi_out", C.c_void_p), ("S_in", C.c_void_p),
        ("S_out", C.c_void_p), ("wall", Wall3D), ("cells", C.c_void_p),
        ("global_flags", C.c_void_p), ("work_cursor", C.c_void_p), ("layout", Layout3D),
        ("N", C.c_int), ("B", C.c_int), ("dt", C.c_float), ("V0", C.c_double),
        ("volume_scale", C.c_double), ("bulk_scale", C.c_float),
        ("interaction_coeff", C.c_float), ("compute_surface", C.c_uint8),
        ("selection", Selection3D), ("tile_pass", C.c_int),
        ("exchange_region", ExchangeRegion3D), ("storage", Storage3D),
    ]


class Vec3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class InitArgs3D(C.Structure):
    _fields_ = [("phi_even", C.c_void_p), ("phi_odd", C.c_void_p), ("cells", C.c_void_p),
                ("centres", C.c_void_p), ("N", C.c_int), ("B", C.c_int), ("layout", Layout3D),
                ("lambda_", C.c_float), ("seed_radius", C.c_float), ("storage", Storage3D)]


class ScatterArgs3D(C.Structure):
    _fields_ = [("phi", C.c_void_p), ("cells", C.c_void_p), ("S", C.c_void_p),
                ("global_flags", C.c_void_p), ("layout", Layout3D), ("N", C.c_int),
                ("B", C.c_int), ("selection", Selection3D), ("storage", Storage3D)]


class Params3D(C.Structure):
    _fields_ = [
        ("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("boundary_flags", C.c_uint32),
        ("num_cells", C.c_int), ("B", C.c_int),
        ("dt", C.c_double), ("lambda_", C.c_double), ("target_radius", C.c_double),
        ("kappa", C.c_double), ("mu", C.c_double), ("xi", C.c_double), ("tau", C.c_double),
        ("v_A", C.c_double), ("gamma", C.c_double), ("v_A_sigma", C.c_double),
        ("aging_time", C.c_double), ("wall_kappa", C.c_double), ("wall_width", C.c_double),
        ("channel_height", C.c_int), ("channel_padding", C.c_int),
        ("seed", C.c_uint64), ("polarity_seed", C.c_uint64), ("full_moment_every", C.c_int),
        ("gamma_soft", C.c_double), ("soft_fraction", C.c_double), ("phi_storage", C.c_int),
    ]


for _cls, _size in ((Cell3D, 256), (Layout3D, 20), (MeasureArgs3D, 168), (UpdateArgs3D, 208),
                    (InitArgs3D, 72), (ScatterArgs3D, 88), (Vec3, 24)):
    assert C.sizeof(_cls) == _size, (_cls.__name__, C.sizeof(_cls))
assert CELL3D_DTYPE.itemsize == 256

P = C.c_void_p
I = C.c_int
_abi._SIGS.update({
    "pfb3d_measure_cells_only": (I, [C.POINTER(MeasureArgs3D), P]),
    "pfb3d_apply_cell_motion": (I, [C.POINTER(MeasureArgs3D), P]),
    "pfb3d_measure_cells": (I, [C.POINTER(MeasureArgs3D), P]),
    "pfb3d_update": (I, [C.POINTER(UpdateArgs3D), P]),
    "pfb3d_step_fused": (I, [C.POINTER(MeasureArgs3D), C.POINTER(UpdateArgs3D), P]),
    "pfb3d_next_brick_edge": (I, [I, I]),
    "pfb3d_shrink_brick_edge": (I, [I, I, P, P]),
    "pfb3d_measure_promoted": (I, [C.POINTER(MeasureArgs3D), P, P, I, I, P]),
    "pfb3d_update_promoted": (I, [C.POINTER(UpdateArgs3D), P, P, P, I, I, P]),
    "pfb3d_scatter_promoted": (I, [C.POINTER(ScatterArgs3D), P, P, I, I, P]),
    "pfb3d_repair_promoted_after_fatal": (I, [C.POINTER(UpdateArgs3D), P, P, P, I, I, P]),
    "pfb3d_check_promoted_crops": (I, [P, P, P, P, I, I, P]),
    "pfb3d_step_cluster": (I, [I]),
    "pfb3d_device_status": (I, [C.POINTER(C.c_uint), I]),
    "pfb3d_clear_S": (I, [P, C.POINTER(Layout3D), P]),
    "pfb3d_repair_after_fatal": (I, [C.POINTER(UpdateArgs3D), P]),
    "pfb3d_finalize_origins": (I, [P, I, P, P]),
    "pfb3d_restore_cells_after_fatal": (I, [P, P, I, P, P, P]),
    "pfb3d_advance_step": (I, [P, P, P]),
    "pfb3d_initialize_spheres": (I, [C.POINTER(InitArgs3D), P]),
    "pfb3d_scatter_current": (I, [C.POINTER(ScatterArgs3D), P]),
    "pfb3d_calibrate_seed_radius": (I, [C.c_double, C.c_double, I, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double)]),
    "pfb3d_automatic_brick_edge": (I, [C.c_double, C.c_double]),
    "pfb3d_initial_polarity": (None, [C.c_int64, C.c_uint64, I, C.POINTER(C.c_double)]),
    "pfb3d_initial_active_speed": (C.c_double, [C.c_int64, C.c_uint64, C.c_double, C.c_double]),
    "pfb3d_soft_membership": (I, [I, C.c_double, C.c_uint64, C.c_void_p]),
    "pfb3d_tumble": (I, [C.c_uint64, C.c_int64, C.c_uint64, C.c_double, I,
                         C.POINTER(C.c_double)]),
    "pfb_sim3d_create": (P, [C.POINTER(Params3D), P, I]),
    "pfb_sim3d_create_from_state": (P, [C.POINTER(Params3D), P, P, C.c_longlong, I]),
    "pfb_sim3d_create_ex": (P, [C.POINTER(Params3D), P, I, I, I]),
    "pfb_sim3d_create_from_state_ex": (P, [C.POINTER(Params3D), P, P, C.c_longlong, I, I, I]),
    "pfb_sim3d_memory_mode": (I, [P]),
    "pfb_sim3d_scratch_slots": (I, [P]),
    "pfb3d_update_inplace": (I, [C.POINTER(UpdateArgs3D), P, I, P]),
    "pfb_sim3d_measure_current": (I, [P]),
    "pfb_sim3d_measure_wall": (I, [P]),
    "pfb_sim3d_verify": (I, [P, C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                             C.POINTER(C.c_ulonglong)]),
    "pfb_sim3d_boundary_open": (I, [P, C.c_char_p, I, C.c_longlong, I]),
    "pfb_sim3d_boundary_capture": (I, [P]),
    "pfb_sim3d_boundary_close": (I, [P, I]),
    "pfb_sim3d_destroy": (None, [P]),
    "pfb_sim3d_advance": (I, [P, I]),
    "pfb_sim3d_set_fused": (I, [P, I]),
    "pfb_sim3d_fused": (I, [P]),
    "pfb_sim3d_set_graph": (I, [P, I]),
    "pfb_sim3d_set_order": (I, [P, I]),
    "pfb_sim3d_packed_words": (I, [P, C.POINTER(C.c_ulonglong)]),
    "pfb_sim3d_get_packed": (I, [P, P]),
    "pfb_sim3d_promoted_count": (I, [P]),
    "pfb_sim3d_max_edge": (I, [P]),
    "pfb_sim3d_recoveries": (C.c_longlong, [P]),
    "pfb_sim3d_sync": (I, [P]),
    "pfb_sim3d_brick": (I, [P]),
    "pfb_sim3d_step": (C.c_longlong, [P]),
    "pfb_sim3d_get_cells": (I, [P, P]),
    "pfb_sim3d_get_phi": (I, [P, P]),
    "pfb_sim3d_get_S": (I, [P, P]),
    "pfb_sim3d_get_flags": (I, [P, P]),
    "pfb_sim3d_layout": (I, [P, C.POINTER(Layout3D)]),
    "pfb_sim3d_update_args": (I, [P, C.POINTER(UpdateArgs3D)]),
    "pfb_sim3d_measure_args": (I, [P, C.POINTER(MeasureArgs3D)]),
    "pfb_sim3d_stream": (P, [P]),
    "pfb_sim3d_bench": (I, [P, I, I, C.POINTER(C.c_double)]),
})
