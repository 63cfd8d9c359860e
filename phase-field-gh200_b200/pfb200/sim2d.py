"""Python face of the 2D host driver (the reference's ``Sim``,
reference include/sim.cuh:58-152) over the C ABI.

Everything here is a thin ctypes call into ``libpfb200.so``; the device work is
the sm_100a kernels in ``csrc/``. Parameter defaults are the reference's
``SimParams`` defaults (reference include/params.cuh:499-530).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, fields

import numpy as np

from ._abi import (CELL_DTYPE, FATAL_FLAGS, FLAG_COUNT, FLAG_NAMES, TILE_AREA, TRAJ_DTYPE,
                   Params2D, StepArgs2D, check, lib, ptr)


@dataclass
class SimParams2D:
    """Model and run parameters of the 2D solver (reference SimParams)."""

    L: int = 0
    num_cells: int = 288
    dt: float = 0.01
    lambda_: float = 7.0
    target_radius: float = 49.0
    kappa: float = 10.0
    mu: float = 1.0
    xi: float = 1500.0
    tau: float = 1.0e4
    v_A: float = 1.0e-2
    gamma_normal: float = 1.0
    gamma_cancer: float = 0.35
    cancer_fraction: float = 0.0
    v_A_sigma: float = 0.0
    phase_field_mobility: float = 0.5
    seed: int = 1234
    polarity_seed: int = 0
    full_moment_every: int = 100
    phi_storage: int = 0  # 0 binary32, 1 binary16, 2 bfloat16 pools

    def to_c(self) -> Params2D:
        p = Params2D()
        for f in fields(self):
            setattr(p, f.name, getattr(self, f.name))
        return p

    @property
    def area0(self) -> float:
        return math.pi * self.target_radius * self.target_radius

    def validate(self) -> None:
        """The checks of the reference's validate() that concern the update
        (reference include/params.cuh:596-722); raises ValueError."""
        if self.L < 144:
            raise ValueError(f"domain side {self.L} is below the class-0 window 144")
        if self.num_cells <= 0:
            raise ValueError("num_cells must be positive")
        for name in ("lambda_", "target_radius", "dt", "xi", "tau"):
            v = getattr(self, name)
            if not (math.isfinite(v) and v > 0):
                raise ValueError(f"{name} must be finite and positive")
        if not (self.kappa >= 0 and self.mu >= 0 and self.v_A >= 0):
            raise ValueError("kappa, mu, v_A must be non-negative")
        gmax = max(self.gamma_normal, self.gamma_cancer)
        cfl = self.dt * gmax * (self.phase_field_mobility / 0.5) * (40.0 / 6.0)
        if cfl >= 1.0:
            raise ValueError(f"dt*(M/M0)*gamma*laplacian_bound = {cfl:.4f} >= 1")


def domain_side_for(n: int, radius: float, rho: float) -> int:
    return int(lib().pfb_domain_side_for(n, radius, rho))


def palmieri_centres(n: int, side: float, min_sep: float, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Sequential periodic placement with minimum separation ``min_sep``
    (reference include/palmieri_initializer.hpp:66-103)."""
    x = np.zeros(n, np.float32)
    y = np.zeros(n, np.float32)
    check(lib().pfb_palmieri_centres(n, float(side), float(min_sep), seed, ptr(x), ptr(y)),
          "palmieri_centres")
    return x, y


def grid_jitter_centres(n: int, side: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Default grid-and-jitter centres (reference src/sim.cu:107-129)."""
    x = np.zeros(n, np.float32)
    y = np.zeros(n, np.float32)
    check(lib().pfb_grid_jitter_centres(n, side, seed, ptr(x), ptr(y)), "grid_jitter")
    return x, y


def step_coefficients(p: SimParams2D) -> StepArgs2D:
    a = StepArgs2D()
    pc = p.to_c()
    check(lib().pfb_fill_coefficients2d(C.byref(pc), C.byref(a)), "fill_coefficients2d")
    return a


def flags_report(flags: np.ndarray) -> dict[str, int]:
    return {FLAG_NAMES[i]: int(flags[i]) for i in range(FLAG_COUNT) if flags[i]}


def fatal(flags: np.ndarray) -> bool:
    return any(int(flags[i]) for i in FATAL_FLAGS)


class Sim2D:
    """Device-resident 2D simulation driven through the C ABI."""

    def __init__(self, params: SimParams2D, cx=None, cy=None, *, device: int = 0,
                 cells: np.ndarray | None = None, phi: np.ndarray | None = None,
                 step: int = 0, cluster: int = 2, use_graph: bool = True, variant: int = 0):
        params.validate()
        self.params = params
        self._pc = params.to_c()
        L = lib()
        if cells is not None:
            cells = np.ascontiguousarray(cells, dtype=CELL_DTYPE)
            phi = np.ascontiguousarray(phi, dtype=np.float32)
            assert cells.shape == (params.num_cells,)
            assert phi.size == params.num_cells * TILE_AREA
            h = L.pfb_sim2d_create_from_state(C.byref(self._pc), ptr(cells), ptr(phi), step,
                                              device)
        else:
            cx = np.ascontiguousarray(cx, dtype=np.float32)
            cy = np.ascontiguousarray(cy, dtype=np.float32)
            assert cx.shape == (params.num_cells,) and cy.shape == (params.num_cells,)
            h = L.pfb_sim2d_create(C.byref(self._pc), ptr(cx), ptr(cy), device)
        if not h:
            raise RuntimeError("pfb_sim2d_create failed: " + L.pfb_last_error().decode())
        self._h = h
        self.set_cluster(cluster)
        check(L.pfb_sim2d_set_variant(h, variant), "set_variant")
        check(L.pfb_sim2d_set_graph(h, 1 if use_graph else 0), "set_graph")

    # ------------------------------------------------------------------ control
    def close(self) -> None:
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                lib().pfb_sim2d_destroy(self._h)
            self._h = None

    @classmethod
    def _view(cls, handle: int, params: "SimParams2D") -> "Sim2D":
        """A non-owning Sim2D over a handle that another object owns."""
        v = cls.__new__(cls)
        v.params = params
        v._pc = params.to_c()
        v._h = handle
        v._owned = False
        return v

    def __del__(self):  # pragma: no cover - interpreter teardown order
        try:
            self.close()
        except Exception:
            pass

    def set_variant(self, variant: int) -> None:
        """0/1: non-returning scatter with exact per-bin overflow detection;
        2: returning scatter that tests every add. Results are identical."""
        check(lib().pfb_sim2d_set_variant(self._h, variant), "set_variant")

    def scatter_recounts(self) -> int:
        """Bins recounted exactly so far (their bound reached 2^32)."""
        out = C.c_uint(0)
        check(lib().pfb_sim2d_scatter_recounts(self._h, C.byref(out)), "scatter_recounts")
        return int(out.value)

    def set_cluster(self, k: int) -> None:
        check(lib().pfb_sim2d_set_cluster(self._h, k), "set_cluster")

    def set_visit_order(self, morton: bool) -> None:
        """Visit the cells in Morton order of their centroids, re-sorted every
        sixth step (reference --morton); results do not change."""
        check(lib().pfb_sim2d_set_visit_order(self._h, 1 if morton else 0), "set_visit_order")

    def visit_order(self) -> np.ndarray:
        out = np.zeros(self.params.num_cells, np.uint32)
        check(lib().pfb_sim2d_visit_order(self._h, out.ctypes.data), "visit_order")
        return out

    def advance(self, steps: int) -> None:
        check(lib().pfb_sim2d_advance(self._h, steps), "advance")

    def sync(self) -> None:
        check(lib().pfb_sim2d_sync(self._h), "sync")

    def bench(self, warmup: int, steps: int) -> float:
        ms = C.c_double(0.0)
        check(lib().pfb_sim2d_bench(self._h, warmup, steps, C.byref(ms)), "bench")
        return ms.value

    # ------------------------------------------------------------------ state
    @property
    def step(self) -> int:
        return int(lib().pfb_sim2d_step(self._h))

    @property
    def side(self) -> int:
        return int(lib().pfb_sim2d_side(self._h))

    @property
    def pitch(self) -> int:
        return int(lib().pfb_sim2d_pitch(self._h))

    @property
    def num_cells(self) -> int:
        return int(lib().pfb_sim2d_num_cells(self._h))

    @property
    def stream(self) -> int:
        return int(lib().pfb_sim2d_stream(self._h) or 0)

    def cells(self) -> np.ndarray:
        out = np.zeros(self.num_cells, CELL_DTYPE)
        check(lib().pfb_sim2d_get_cells(self._h, ptr(out)), "get_cells")
        return out

    def phi(self) -> np.ndarray:
        out = np.zeros((self.num_cells, 288, 288), np.float32)
        check(lib().pfb_sim2d_get_phi(self._h, ptr(out)), "get_phi")
        return out

    def S(self) -> np.ndarray:
        out = np.zeros((self.side, self.pitch), np.uint32)
        check(lib().pfb_sim2d_get_S(self._h, ptr(out)), "get_S")
        return out

    def flags(self) -> np.ndarray:
        out = np.zeros(FLAG_COUNT, np.uint32)
        check(lib().pfb_sim2d_get_flags(self._h, ptr(out)), "get_flags")
        return out

    def traj(self) -> np.ndarray:
        out = np.zeros(self.num_cells, TRAJ_DTYPE)
        check(lib().pfb_sim2d_pack_traj(self._h, ptr(out)), "pack_traj")
        return out

    def advance_record(self, steps: int, every: int, ring: np.ndarray) -> None:
        """Advance `steps` steps, copying the trajectory records of every
        `every`-th step into frame k % len(ring) of `ring` (a TRAJ_DTYPE array
        of shape (frames, num_cells), ideally in page-locked memory) without a
        host wait; the frames are valid after sync()."""
        if ring.dtype != TRAJ_DTYPE or ring.ndim != 2 or ring.shape[1] != self.num_cells or \
                not ring.flags.c_contiguous:
            raise ValueError("ring must be a C-contiguous (frames, num_cells) TRAJ_DTYPE array")
        check(lib().pfb_sim2d_advance_record(self._h, steps, every, ptr(ring), ring.shape[0]),
              "advance_record")

    def set_state(self, cells: np.ndarray, phi: np.ndarray, step: int) -> None:
        cells = np.ascontiguousarray(cells, dtype=CELL_DTYPE)
        phi = np.ascontiguousarray(phi, dtype=np.float32)
        check(lib().pfb_sim2d_set_state(self._h, ptr(cells), ptr(phi), step), "set_state")

    def save(self) -> None:
        """In-memory device checkpoint of the current step."""
        check(lib().pfb_sim2d_save(self._h), "save")

    def restore(self) -> None:
        check(lib().pfb_sim2d_restore(self._h), "restore")

    def velocity_open(self, path, spatial_stride: int = 100, dense_start: int = 10000,
                      reference: bool = False) -> None:
        """Start a PFVMOM4 velocity-component recording in a new file
        (writes the header and the frame of the current step)."""
        check(lib().pfb_sim2d_velocity_open(self._h, str(path).encode(), spatial_stride,
                                            dense_start, 1 if reference else 0), "velocity_open")

    def velocity_capture(self) -> None:
        check(lib().pfb_sim2d_velocity_capture(self._h), "velocity_capture")

    def velocity_close(self) -> None:
        check(lib().pfb_sim2d_velocity_close(self._h), "velocity_close")

    def verify(self) -> tuple[float, float, int]:
        """(max relative volume error, max |phi| outside the windows, max
        aggregate word) of the current state."""
        rel, out, smax = C.c_double(), C.c_float(), C.c_uint32()
        check(lib().pfb_sim2d_verify(self._h, C.byref(rel), C.byref(out), C.byref(smax)), "verify")
        return rel.value, out.value, smax.value

    def boundary_open(self, path, interval: int, compress: bool = False) -> None:
        """Start a PFB boundary recording in a new file (header only)."""
        check(lib().pfb_sim2d_boundary_open(self._h, str(path).encode(), interval,
                                            1 if compress else 0), "boundary_open")

    def boundary_capture(self) -> None:
        check(lib().pfb_sim2d_boundary_capture(self._h), "boundary_capture")

    def boundary_close(self) -> None:
        check(lib().pfb_sim2d_boundary_close(self._h), "boundary_close")

    def residual_step(self) -> tuple[float, float]:
        """Advance one step; (max, rms) of |dphi / dt| over that step."""
        linf, rms = C.c_double(), C.c_double()
        check(lib().pfb_sim2d_residual_step(self._h, C.byref(linf), C.byref(rms)), "residual")
        return linf.value, rms.value

    def step_args(self) -> StepArgs2D:
        a = StepArgs2D()
        check(lib().pfb_sim2d_step_args(self._h, C.byref(a)), "step_args")
        return a


def window_view(phi: np.ndarray, cells: np.ndarray, n: int) -> np.ndarray:
    """Active window of cell n (rows y, cols x) inside its 288^2 tile."""
    from ._abi import CLASSES
    wx, wy, tx0, ty0 = CLASSES[int(cells["cls"][n])]
    return phi[n, ty0:ty0 + wy, tx0:tx0 + wx]


def world_field(phi: np.ndarray, cells: np.ndarray, n: int, L: int) -> np.ndarray:
    """Cell n's phi scattered onto the periodic L x L lattice (world frame)."""
    w = window_view(phi, cells, n)
    out = np.zeros((L, L), np.float64)
    gy = (int(cells["gy0"][n]) + np.arange(w.shape[0])) % L
    gx = (int(cells["gx0"][n]) + np.arange(w.shape[1])) % L
    out[np.ix_(gy, gx)] = w
    return out
