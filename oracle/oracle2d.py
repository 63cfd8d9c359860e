"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py). ctypes access to:

* ``oracle/_build/liboracle2d.so``: the CPU restatement of the reference's 2D
  step (``pf2d_oracle.cpp``), f32 and f64 modes;
* ``oracle/_ref/libref2d.so``: the reference's own CUDA step kernel compiled in
  place for sm_100a (``ref2d_shim.cu``), when it was built.

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

from pfb200._abi import CELL_DTYPE, Params2D, StepArgs2D  # noqa: E402

ORACLE_SO = HERE / "_build" / "liboracle2d.so"
REF_SO = HERE / "_ref" / "libref2d.so"
REF_BIN = HERE / "_ref" / "cell_gh200"

_O = None
_R = None
P = C.c_void_p


def build() -> None:
    """Compile the CPU restatement (and, when the reference tree is present,
    the reference in place)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    subprocess.run(["make", "-s", "-C", str(HERE), "ref"], check=True)


def olib() -> C.CDLL:
    global _O
    if _O is None:
        if not ORACLE_SO.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
        L = C.CDLL(str(ORACLE_SO))
        L.oracle_philox4x32_10.argtypes = [C.c_uint32] * 6 + [C.POINTER(C.c_uint32)]
        L.oracle_philox4x32_10.restype = None
        L.oracle_u53.argtypes = [C.c_uint32, C.c_uint32]
        L.oracle_u53.restype = C.c_double
        L.oracle_q_of.argtypes = [C.c_float]
        L.oracle_q_of.restype = C.c_uint32
        L.oracle_rhs_f32.argtypes = [C.c_float] * 12
        L.oracle_rhs_f32.restype = C.c_float
        L.oracle_coefficients_f32.argtypes = [C.c_float] * 5 + [C.POINTER(C.c_float)]
        L.oracle_coefficients_f32.restype = None
        L.oracle_coefficients_f64.argtypes = [C.c_double] * 5 + [C.POINTER(C.c_double)]
        L.oracle_coefficients_f64.restype = None
        L.oracle_step2d_f32.argtypes = [C.POINTER(StepArgs2D), C.c_int]
        L.oracle_step2d_f32.restype = C.c_int
        L.oracle_sim_create.argtypes = [C.POINTER(Params2D), P, P, C.c_longlong, C.c_int]
        L.oracle_sim_create.restype = P
        L.oracle_sim_destroy.argtypes = [P, C.c_int]
        L.oracle_sim_destroy.restype = None
        L.oracle_sim_advance.argtypes = [P, C.c_int, C.c_longlong, C.c_int]
        L.oracle_sim_advance.restype = None
        L.oracle_sim_step.argtypes = [P, C.c_int]
        L.oracle_sim_step.restype = C.c_longlong
        for name in ("oracle_sim_get_cells", "oracle_sim_get_velocity", "oracle_sim_get_phi",
                     "oracle_sim_get_S", "oracle_sim_get_flags"):
            f = getattr(L, name)
            f.argtypes = [P, C.c_int, P]
            f.restype = None
        L.oracle_init_state2d.argtypes = [C.POINTER(Params2D), P, P, P, P]
        L.oracle_init_state2d.restype = None
        L.oracle_scatter_all2d.argtypes = [P, P, C.c_int, C.c_int, C.c_int, P, P]
        L.oracle_scatter_all2d.restype = None
        L.oracle_palmieri_centres.argtypes = [C.c_int, C.c_double, C.c_double, C.c_ulonglong,
                                              P, P]
        L.oracle_palmieri_centres.restype = C.c_int
        L.oracle_ic_theta.argtypes = [C.c_int32, C.c_ulonglong]
        L.oracle_ic_theta.restype = C.c_float
        L.oracle_ic_v_A.argtypes = [C.c_int32, C.c_ulonglong, C.c_double, C.c_double]
        L.oracle_ic_v_A.restype = C.c_double
        L.oracle_fresh_cells2d.argtypes = [C.POINTER(Params2D), P]
        L.oracle_fresh_cells2d.restype = None
        _O = L
    return _O


def ref_available() -> bool:
    return REF_SO.exists()


def rlib() -> C.CDLL:
    """The reference's own step kernel (sm_100a build)."""
    global _R
    if _R is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} was not built")
        L = C.CDLL(str(REF_SO))
        L.ref2d_launch_step.argtypes = [C.POINTER(StepArgs2D), C.c_int, P]
        L.ref2d_launch_step.restype = C.c_int
        L.ref2d_grid.argtypes = [C.c_int]
        L.ref2d_grid.restype = C.c_int
        L.ref2d_configure.argtypes = []
        L.ref2d_configure.restype = C.c_int
        L.ref2d_scatter_all.argtypes = [P, P, P, P, C.c_int, C.c_int, C.c_int, P, P]
        L.ref2d_scatter_all.restype = C.c_int
        L.ref2d_ic_theta.argtypes = [C.c_int32, C.c_ulonglong]
        L.ref2d_ic_theta.restype = C.c_float
        L.ref2d_ic_v_A.argtypes = [C.c_int32, C.c_ulonglong, C.c_double, C.c_double]
        L.ref2d_ic_v_A.restype = C.c_double
        L.ref2d_init_tiles.argtypes = [P, P, P, P, C.c_int, C.c_int, P, P, C.c_float, C.c_float,
                                       P]
        L.ref2d_init_tiles.restype = C.c_int
        L.ref2d_init_moments.argtypes = [P, P, P, C.c_int, P]
        L.ref2d_init_moments.restype = C.c_int
        _R = L
    return _R


def _p(a):
    return None if a is None else a.ctypes.data


def philox(c, k) -> list[int]:
    out = (C.c_uint32 * 4)()
    olib().oracle_philox4x32_10(*[int(v) for v in c], *[int(v) for v in k], out)
    return list(out)


def coefficients(lam, kappa, xi, mu, target, f64: bool):
    if f64:
        out = (C.c_double * 6)()
        olib().oracle_coefficients_f64(lam, kappa, xi, mu, target, out)
    else:
        out = (C.c_float * 6)()
        olib().oracle_coefficients_f32(lam, kappa, xi, mu, target, out)
    return list(out)


def palmieri_centres(n: int, side: float, min_sep: float, seed: int):
    """Sequential periodic placement (reference include/palmieri_initializer.hpp:66-103)."""
    x = np.zeros(n, np.float32)
    y = np.zeros(n, np.float32)
    rc = olib().oracle_palmieri_centres(n, float(side), float(min_sep), seed, _p(x), _p(y))
    if rc:
        raise RuntimeError("oracle placement did not terminate")
    return x, y


def fresh_cells(params_c: Params2D) -> np.ndarray:
    """Cell records of a fresh start (reference src/sim.cu:136-143, 324-340)."""
    cells = np.zeros(params_c.num_cells, CELL_DTYPE)
    olib().oracle_fresh_cells2d(C.byref(params_c), _p(cells))
    return cells


def init_state(params_c: Params2D, cx: np.ndarray, cy: np.ndarray, cells: np.ndarray):
    """Seed tanh disks on the host (binary32, reference k_init_tiles math)."""
    N = params_c.num_cells
    phi = np.zeros((N, 288, 288), np.float32)
    cells = np.ascontiguousarray(cells.copy())
    olib().oracle_init_state2d(C.byref(params_c), _p(np.ascontiguousarray(cx, np.float32)),
                               _p(np.ascontiguousarray(cy, np.float32)), _p(cells), _p(phi))
    return cells, phi


def scatter_all(phi, cells, L, P):
    S = np.zeros((L, P), np.uint32)
    flags = np.zeros(8, np.uint32)
    olib().oracle_scatter_all2d(_p(phi), _p(cells), len(cells), L, P, _p(S), _p(flags))
    return S, flags


class OracleSim:
    """Whole-run CPU driver (slot scheme of the reference's Sim)."""

    def __init__(self, params_c: Params2D, cells: np.ndarray, phi: np.ndarray, step: int = 0,
                 f64: bool = False):
        self.f64 = int(f64)
        self.N = params_c.num_cells
        self.L = params_c.L
        self.P = 32 * ((self.L + 31) // 32)
        self._pc = params_c
        cells = np.ascontiguousarray(cells, dtype=CELL_DTYPE)
        phi = np.ascontiguousarray(phi, dtype=np.float32)
        self._h = olib().oracle_sim_create(C.byref(self._pc), _p(cells), _p(phi), step, self.f64)
        if not self._h:
            raise RuntimeError("oracle_sim_create failed")

    def close(self):
        if self._h:
            olib().oracle_sim_destroy(self._h, self.f64)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _handle(self):
        if not self._h:
            raise RuntimeError("the oracle simulation was closed")
        return self._h

    def advance(self, steps: int, threads: int = 0):
        olib().oracle_sim_advance(self._handle(), self.f64, steps, threads)

    @property
    def step(self) -> int:
        return int(olib().oracle_sim_step(self._handle(), self.f64))

    def cells(self) -> np.ndarray:
        out = np.zeros(self.N, CELL_DTYPE)
        olib().oracle_sim_get_cells(self._handle(), self.f64, _p(out))
        return out

    def velocity(self) -> np.ndarray:
        out = np.zeros((self.N, 2), np.float64)
        olib().oracle_sim_get_velocity(self._handle(), self.f64, _p(out))
        return out

    def phi(self) -> np.ndarray:
        out = np.zeros((self.N, 288, 288), np.float64)
        olib().oracle_sim_get_phi(self._handle(), self.f64, _p(out))
        return out

    def S(self) -> np.ndarray:
        out = np.zeros((self.L, self.P), np.uint32)
        olib().oracle_sim_get_S(self._handle(), self.f64, _p(out))
        return out

    def flags(self) -> np.ndarray:
        out = np.zeros(8, np.uint32)
        olib().oracle_sim_get_flags(self._handle(), self.f64, _p(out))
        return out
