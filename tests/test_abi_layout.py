"""The C-ABI library loads without a GPU, exports every entry point that
include/pfb200.h declares, and its records have the reference's layout
(reference include/kernels.cuh:27-57 CellState, :74-116 StepArgs)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

import pfb200
from pfb200._abi import CELL_DTYPE, Cell2D, Params2D, StepArgs2D, TrajCell2D

INCLUDE = Path(__file__).resolve().parent.parent / "include"
HEADERS = sorted(INCLUDE.glob("*.h"))


def declared_functions(paths=HEADERS):
    names = set()
    for path in paths:
        text = re.sub(r"/\*.*?\*/", "", path.read_text(), flags=re.S)
        names.update(re.findall(r"\b(pfb[0-9a-z_]*_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "pfb_step2d_launch" in names and "pfb_sim2d_create" in names
    assert "pfb3d_update" in names and "pfb_sim3d_create" in names
    assert len(names) >= 70


def test_library_exports_every_declared_symbol():
    L = pfb200.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) <= set(pfb200.exported_symbols())


def test_record_sizes_match_library():
    L = pfb200.lib()
    assert L.pfb_sizeof(0) == 192 == C.sizeof(Cell2D) == CELL_DTYPE.itemsize
    assert L.pfb_sizeof(1) == 216 == C.sizeof(StepArgs2D)
    assert L.pfb_sizeof(2) == C.sizeof(Params2D)
    assert L.pfb_sizeof(3) == 48 == C.sizeof(TrajCell2D)


def test_cell_record_offsets():
    # The reference pins these with static_asserts (include/kernels.cuh:53-57).
    assert Cell2D.advection.offset == 128
    assert Cell2D.reserved.offset == 120
    assert Cell2D.M_pf.offset == 188
    for name, (dt, off) in CELL_DTYPE.fields.items():
        if name.startswith("adv_"):
            continue
        assert getattr(Cell2D, name).offset == off, name


def test_step_args_offsets():
    expect = {"phi_in": 0, "flags": 96, "moments": 104, "physical_dt": 112, "N": 120,
              "parity_out": 132, "dt": 136, "A0": 144, "vol_scale": 152, "bulk_scale": 160,
              "mot_coeff": 168, "seed": 176, "polarity_seed": 184, "p_tumble": 192,
              "full_moment_every": 200, "clear_ahead_words": 208}
    for k, v in expect.items():
        assert getattr(StepArgs2D, k).offset == v, k


def test_launcher_rejects_bad_arguments_without_touching_a_device():
    L = pfb200.lib()
    assert L.pfb_step2d_launch(None, 4, None) == -1
    a = StepArgs2D()
    assert L.pfb_step2d_launch(C.byref(a), 4, None) == -1  # null buffers
    assert b"null" in L.pfb_last_error()
    assert L.pfb_step2d_grid(64, 0) == 128  # default clusters of 2
    assert L.pfb_step2d_grid(64, 8) == 512
    assert L.pfb_step2d_grid(64, 3) == -1


def test_coefficients_match_reference_defaults():
    p = pfb200.SimParams2D(L=512, num_cells=64, target_radius=12.0)
    a = pfb200.step_coefficients(p)
    assert a.dt == np.float32(0.01)
    assert abs(a.A0 - np.pi * 144.0) < 1e-12
    assert a.bulk_scale == np.float32(30.0 / 49.0)
    assert a.rep_coeff == np.float32(600.0 / 49.0)
    assert a.mot_coeff == np.float32((600.0 / 49.0) / 1500.0)
    assert a.p_tumble == -np.expm1(-0.01 / 1e4)
    assert a.polarity_seed == 1234


def test_3d_record_layouts():
    # reference include/pf3d/kernels.cuh:132-137 static_asserts and the
    # measured offsets of MeasureArgs3D / UpdateArgs3D
    from pfb200._abi3d import (Cell3D, InitArgs3D, MeasureArgs3D, ScatterArgs3D,
                               UpdateArgs3D)
    assert C.sizeof(Cell3D) == 256 and Cell3D.storage_edge.offset == 192
    assert Cell3D.V.offset == 128 and Cell3D.pending_shift_x.offset == 112
    assert C.sizeof(MeasureArgs3D) == 168 and MeasureArgs3D.apply_tumble.offset == 140
    assert MeasureArgs3D.selection.offset == 144 and MeasureArgs3D.storage.offset == 160
    assert C.sizeof(UpdateArgs3D) == 208 and UpdateArgs3D.tile_pass.offset == 152
    assert UpdateArgs3D.exchange_region.offset == 156 and UpdateArgs3D.storage.offset == 200
    assert C.sizeof(InitArgs3D) == 72 and C.sizeof(ScatterArgs3D) == 88


def test_3d_launchers_reject_bad_arguments_without_touching_a_device():
    from pfb200._abi3d import MeasureArgs3D, UpdateArgs3D
    L = pfb200.lib()
    assert L.pfb3d_update(None, None) == -1
    u = UpdateArgs3D()
    assert L.pfb3d_update(C.byref(u), None) < 0
    u.B, u.N = 64, 4
    u.layout.nx = u.layout.ny = u.layout.nz = 256
    u.layout.pitch_x = 256
    u.layout.boundary_flags = 0x7
    assert L.pfb3d_update(C.byref(u), None) == -1  # null buffers
    u.tile_pass = 1
    assert L.pfb3d_update(C.byref(u), None) == -3  # boundary-first pass unsupported
    m = MeasureArgs3D()
    m.B, m.N = 64, 4
    m.layout = u.layout
    m.storage.z_cap = 8
    assert L.pfb3d_measure_cells_only(C.byref(m), None) == -3  # compact storage


def test_conv_pipeline_modes():
    """pfb_conv_set_pipeline takes 0, 1 (default) and 2 and rejects the rest
    without touching a device."""
    L = pfb200.lib()
    try:
        for mode in (0, 2, 1):
            assert L.pfb_conv_set_pipeline(mode) == 0
        assert L.pfb_conv_set_pipeline(3) == -1
        assert L.pfb_conv_set_pipeline(-1) == -1
        assert b"pipeline" in L.pfb_last_error()
    finally:
        L.pfb_conv_set_pipeline(1)
