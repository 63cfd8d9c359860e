"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py). ctypes access to:

* ``oracle/_build/liboracle3d.so``: the CPU restatement of the reference's 3D
  step (``pf3d_oracle.cpp``), f32 and f64 modes;
* ``oracle/_ref/libref3d.so``: the reference's own 3D launchers compiled in
  place for sm_100a (``ref3d_shim.cu``), when built;
* ``oracle/_ref/libref3d_cpu.so``: the reference's dense FP64 one-step,
  seed-radius calibration and Philox draws (``ref3d_cpu_shim.cpp``), when
  built.

Nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
sys.path.insert(0, str(REPO / "phase-field-gh200_b200"))

from pfb200._abi3d import CELL3D_DTYPE, Layout3D  # noqa: E402

ORACLE_SO = HERE / "_build" / "liboracle3d.so"
REF_SO = HERE / "_ref" / "libref3d.so"
REF_CPU_SO = HERE / "_ref" / "libref3d_cpu.so"

_O = None
_R = None
_RC = None
P = C.c_void_p
I = C.c_int
D = C.c_double


def olib() -> C.CDLL:
    global _O
    if _O is None:
        if not ORACLE_SO.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
        L = C.CDLL(str(ORACLE_SO))
        L.oracle3d_step.argtypes = [I, P, P, P, P, P, P, P, C.POINTER(Layout3D), I, I, P, D, D,
                                    D, D, D, D, D, C.c_uint64, C.c_uint64, I, I]
        L.oracle3d_step.restype = I
        L.oracle3d_measure.argtypes = [I, P, P, P, P, C.c_uint64, C.POINTER(Layout3D), I, I, P,
                                       D, D, D, D, D, C.c_uint64, C.c_uint64, I, I, I]
        L.oracle3d_measure.restype = None
        L.oracle3d_scatter.argtypes = [I, P, P, P, P, C.POINTER(Layout3D), I, I]
        L.oracle3d_scatter.restype = None
        L.oracle3d_q32.argtypes = [C.c_float]
        L.oracle3d_q32.restype = C.c_uint32
        _O = L
    return _O


def ref_available() -> bool:
    return REF_SO.exists()


def ref_cpu_available() -> bool:
    return REF_CPU_SO.exists()


def rlib() -> C.CDLL:
    """The reference's own 3D launchers (sm_100a build)."""
    global _R
    if _R is None:
        L = C.CDLL(str(REF_SO))
        for name in ("ref3d_measure_cells_only", "ref3d_apply_cell_motion", "ref3d_update_periodic",
                     "ref3d_repair_after_fatal", "ref3d_initialize_spheres",
                     "ref3d_scatter_current"):
            getattr(L, name).argtypes = [P, P]
            getattr(L, name).restype = I
        L.ref3d_update_tiled.argtypes = [P, I, P]
        L.ref3d_update_tiled.restype = I
        L.ref3d_clear_S.argtypes = [P, P, P]
        L.ref3d_clear_S.restype = I
        L.ref3d_finalize_origins.argtypes = [P, I, P, P]
        L.ref3d_finalize_origins.restype = I
        L.ref3d_restore_cells_after_fatal.argtypes = [P, P, I, P, P]
        L.ref3d_restore_cells_after_fatal.restype = I
        L.ref3d_advance_step.argtypes = [P, P, P]
        L.ref3d_advance_step.restype = I
        _R = L
    return _R


def rclib() -> C.CDLL:
    """The reference's dense FP64 one-step and Philox draws (host build)."""
    global _RC
    if _RC is None:
        L = C.CDLL(str(REF_CPU_SO))
        L.ref3d_cpu_one_step.argtypes = [I, I, P, P, P, P, D, D, D, D, D, D, P, P, P, P]
        L.ref3d_cpu_one_step.restype = I
        L.ref3d_cpu_calibrate.argtypes = [D, D, I, C.POINTER(D), C.POINTER(D)]
        L.ref3d_cpu_calibrate.restype = I
        L.ref3d_cpu_initial_polarity.argtypes = [C.c_int64, C.c_uint64, I, C.POINTER(D)]
        L.ref3d_cpu_initial_polarity.restype = None
        L.ref3d_cpu_initial_speed.argtypes = [C.c_int64, C.c_uint64, D, D]
        L.ref3d_cpu_initial_speed.restype = D
        L.ref3d_cpu_tumble.argtypes = [C.c_uint64, C.c_int64, C.c_uint64, D, I, C.POINTER(D)]
        L.ref3d_cpu_tumble.restype = I
        F = C.POINTER(C.c_float)
        L.ref3d_cpu_palmieri2d.argtypes = [I, D, D, C.c_uint64, F, F]
        L.ref3d_cpu_palmieri2d.restype = I
        L.ref3d_cpu_palmieri3d.argtypes = [I, D, D, C.c_uint64, F, F, F]
        L.ref3d_cpu_palmieri3d.restype = I
        L.ref3d_cpu_channel3d.argtypes = [I, D, I, D, C.c_uint64, F, F, F]
        L.ref3d_cpu_channel3d.restype = I
        L.ref3d_cpu_table_hash.argtypes = [I, F, F, F]
        L.ref3d_cpu_table_hash.restype = C.c_uint64
        U = C.POINTER(C.c_uint64)
        L.ref_soft_membership.argtypes = [I, D, C.c_uint64, P]
        L.ref_soft_membership.restype = I
        L.ref_read_table2.argtypes = [C.c_char_p, I, D, D, F, F, U]
        L.ref_read_table2.restype = I
        L.ref_read_relaxed2.argtypes = [C.c_char_p, I, D, I, F, F]
        L.ref_read_relaxed2.restype = I
        L.ref_read_table3.argtypes = [C.c_char_p, I, D, D, F, F, F, U]
        L.ref_read_table3.restype = I
        L.ref_read_channel3.argtypes = [C.c_char_p, I, D, I, D, F, F, F, U]
        L.ref_read_channel3.restype = I
        _RC = L
    return _RC


def _p(a):
    return None if a is None else a.ctypes.data


class OracleState3D:
    """Host copy of a 3D system stepped by the CPU restatement."""

    def __init__(self, params, layout: Layout3D, B: int, cells: np.ndarray, phi: np.ndarray,
                 S: np.ndarray, step: int = 0, f64: bool = False, wall=None):
        self.p = params
        self.L = layout
        self.B = B
        self.f64 = f64
        self.cells = np.ascontiguousarray(cells.copy(), dtype=CELL3D_DTYPE)
        dt = np.float64 if f64 else np.float32
        self.phi = np.ascontiguousarray(phi, dtype=dt).copy()
        self.S = np.ascontiguousarray(S, dtype=np.uint32).copy()
        self.flags = np.zeros(10, np.uint32)
        self.step = np.array([step], np.uint64)
        self.steps_done = 0
        self.wall = None if wall is None else np.ascontiguousarray(wall, dtype=np.float32)
        if f64:
            # the aggregate of the binary64 field: q(phi) of a widened binary32
            # value can differ from the binary32 q by one unit, which the step
            # would count as a negative S_other
            self.S[...] = 0
            olib().oracle3d_scatter(1, _p(self.phi), _p(self.cells), _p(self.S), _p(self.flags),
                                    C.byref(self.L), len(self.cells), B)

    def advance(self, n: int = 1, threads: int = 0) -> list[int]:
        p = self.p
        out = []
        for _ in range(n):
            nxt = np.zeros_like(self.phi)
            S_out = np.zeros_like(self.S)
            full = p.full_moment_every > 0 and self.steps_done % p.full_moment_every == 0
            aging = int(p.aging_time / p.dt + 0.5)
            rc = olib().oracle3d_step(
                1 if self.f64 else 0, _p(self.phi), _p(nxt), _p(self.S), _p(S_out),
                _p(self.cells), _p(self.flags), _p(self.step), C.byref(self.L),
                len(self.cells), self.B, _p(self.wall), p.dt, p.lambda_, p.kappa, p.mu, p.xi,
                p.tau, p.target_radius, p.polarity_seed or p.seed, aging, 1 if full else 0,
                threads)
            self.phi, self.S = nxt, S_out
            self.steps_done += 1
            out.append(rc)
        return out
