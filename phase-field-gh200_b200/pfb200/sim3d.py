"""Python face of the 3D host driver (the reference's ``Sim3D`` step
sequence, reference src/pf3d/sim.cu:1460-1651) over the C ABI of
``include/pfb200_3d.h``. Parameter defaults are the reference's
``SimParams3D`` defaults (reference include/pf3d/params.cuh:257-300)."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, fields

import numpy as np

from ._abi import check, lib, ptr
from ._abi3d import (BOUNDARY_HARD_WALL_CHANNEL, BOUNDARY_PERIODIC_XYZ,
                     BOUNDARY_SUBSTRATE_SLAB, CELL3D_DTYPE, FLAG3D_COUNT, FLAG3D_NAMES, Layout3D,
                     MeasureArgs3D, Params3D, UpdateArgs3D)

GEOMETRIES = {"periodic": BOUNDARY_PERIODIC_XYZ, "slab": BOUNDARY_SUBSTRATE_SLAB,
              "channel": BOUNDARY_HARD_WALL_CHANNEL}


@dataclass
class SimParams3D:
    """Model and run parameters of the 3D driver (reference SimParams3D)."""

    Nx: int = 0
    Ny: int = 0
    Nz: int = 0
    geometry: str = "periodic"
    num_cells: int = 288
    B: int = 0  # 0: automatic brick edge
    dt: float = 0.01
    lambda_: float = 7.0
    target_radius: float = 49.0
    kappa: float = 10.0
    mu: float = 1.0
    xi: float = 1500.0
    tau: float = 1.0e4
    v_A: float = 1.0e-2
    gamma: float = 1.0
    v_A_sigma: float = 0.0
    aging_time: float = 0.0
    wall_kappa: float = 0.0
    wall_width: float = 0.0
    channel_height: int = 0
    channel_padding: int = 0
    seed: int = 1234
    polarity_seed: int = 0
    full_moment_every: int = 100
    gamma_soft: float = 0.35     # soft cells' stiffness (reference gamma_cancer)
    soft_fraction: float = 0.0   # share of soft identities (reference cancer_fraction)
    phi_storage: int = 0         # base pools: 0 binary32, 1 binary16, 2 bfloat16

    def to_c(self) -> Params3D:
        p = Params3D()
        for f in fields(self):
            if f.name == "geometry":
                p.boundary_flags = GEOMETRIES[self.geometry]
            else:
                setattr(p, f.name, getattr(self, f.name))
        return p

    @property
    def boundary_flags(self) -> int:
        return GEOMETRIES[self.geometry]

    @property
    def volume0(self) -> float:
        v = 4.0 * math.pi * self.target_radius ** 3 / 3.0
        return 0.5 * v if self.geometry == "slab" else v

    def brick(self) -> int:
        return self.B or automatic_brick_edge(self.target_radius, self.lambda_)


def automatic_brick_edge(radius: float, lam: float) -> int:
    return int(lib().pfb3d_automatic_brick_edge(radius, lam))


def calibrate_seed_radius(radius: float, lam: float, edge: int) -> tuple[float, float]:
    s, v = C.c_double(), C.c_double()
    check(lib().pfb3d_calibrate_seed_radius(radius, lam, edge, C.byref(s), C.byref(v)),
          "calibrate_seed_radius")
    return s.value, v.value


def domain_side_for(n: int, radius: float, rho: float) -> int:
    """Periodic cube side holding n spheres at volume fraction rho
    (reference include/pf3d/params.cuh:214-223)."""
    return int(math.ceil(((n * 4.0 * math.pi * radius ** 3 / 3.0) / rho) ** (1.0 / 3.0)))


def sequential_centres(n: int, side: float, min_sep: float, seed: int, *, height: float = 0.0,
                       z_margin: float = 0.0, planar_z: float | None = None,
                       first_at_centre: bool = False,
                       max_tries: int = 1_000_000) -> np.ndarray:
    """Seeded random sequential placement with a minimum periodic separation
    (periodic in x, y; in z too unless `height` bounds it). Returns (n, 3).
    first_at_centre puts cell 0 at the box centre, the convention of the
    reference's periodic initialiser and centre tables
    (reference include/pf3d/palmieri_initializer.hpp:149-154)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 3))
    k = 0
    if first_at_centre and n:
        out[0] = 0.5 * side
        k = 1
    tries = 0
    while k < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"placed only {k} of {n} centres")
        c = rng.random(3) * side
        if planar_z is not None:
            c[2] = planar_z
        elif height > 0.0:
            c[2] = z_margin + rng.random() * (height - 2.0 * z_margin)
        if k:
            d = out[:k] - c
            d[:, :2] -= side * np.round(d[:, :2] / side)
            if planar_z is None and height <= 0.0:
                d[:, 2] -= side * np.round(d[:, 2] / side)
            if np.min(np.einsum("ij,ij->i", d, d)) < min_sep * min_sep:
                continue
        out[k] = c
        k += 1
    return out


def flags_report3(flags: np.ndarray) -> dict[str, int]:
    return {FLAG3D_NAMES[i]: int(flags[i]) for i in range(FLAG3D_COUNT) if flags[i]}


class Sim3D:
    """Device-resident 3D simulation driven through the C ABI."""

    MEMORY_MODES = {"auto": -1, "throughput": 0, "balanced": 1, "compact": 2}

    def __init__(self, params: SimParams3D, centres: np.ndarray | None = None, *, device: int = 0,
                 cells: np.ndarray | None = None, phi: np.ndarray | None = None, step: int = 0,
                 memory_mode: str = "auto", scratch_slots: int = 0):
        """Fresh start from centres, or a restart from cell records and fields
        (cells, phi) of step `step`: phi is (N, B, B, B) or each cell's field
        packed in cell order (E^3 values for a cell on a promoted cube)."""
        self.params = params
        self._pc = params.to_c()
        if cells is not None:
            self._cells0 = np.ascontiguousarray(cells, dtype=CELL3D_DTYPE)
            self._phi0 = np.ascontiguousarray(phi, dtype=np.float32)
            assert self._cells0.shape == (params.num_cells,)
            h = lib().pfb_sim3d_create_from_state_ex(C.byref(self._pc), ptr(self._cells0),
                                                     ptr(self._phi0), step, device,
                                                     self.MEMORY_MODES[memory_mode], scratch_slots)
            del self._cells0, self._phi0
        else:
            c = np.ascontiguousarray(centres, dtype=np.float64)
            assert c.shape == (params.num_cells, 3)
            h = lib().pfb_sim3d_create_ex(C.byref(self._pc), ptr(c), device,
                                          self.MEMORY_MODES[memory_mode], scratch_slots)
        if not h:
            raise RuntimeError("pfb_sim3d_create failed: " + lib().pfb_last_error().decode())
        self._h = h
        lay = Layout3D()
        check(lib().pfb_sim3d_layout(h, C.byref(lay)), "layout")
        self.layout = lay
        self.B = int(lib().pfb_sim3d_brick(h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pfb_sim3d_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter teardown order
        try:
            self.close()
        except Exception:
            pass

    def advance(self, steps: int) -> None:
        check(lib().pfb_sim3d_advance(self._h, steps), "advance")

    def sync(self) -> None:
        check(lib().pfb_sim3d_sync(self._h), "sync")

    @property
    def fused(self) -> bool:
        """True when a step runs as one fused measure + motion + update launch."""
        return bool(lib().pfb_sim3d_fused(self._h))

    def set_fused(self, fused: bool) -> None:
        check(lib().pfb_sim3d_set_fused(self._h, 1 if fused else 0), "set_fused")

    def set_graph(self, use_graph: bool) -> None:
        check(lib().pfb_sim3d_set_graph(self._h, 1 if use_graph else 0), "set_graph")

    def packed(self) -> np.ndarray:
        """Current fields of all cells packed in cell order, each on its own
        cube (B^3 or E^3 values)."""
        w = C.c_ulonglong(0)
        check(lib().pfb_sim3d_packed_words(self._h, C.byref(w)), "packed_words")
        out = np.zeros(w.value, np.float32)
        check(lib().pfb_sim3d_get_packed(self._h, ptr(out)), "get_packed")
        return out

    def fields(self) -> list[np.ndarray]:
        """Each cell's current field as an (E, E, E) array."""
        cells, flat = self.cells(), self.packed()
        out, off = [], 0
        for e in cells["storage_edge"]:
            e = int(e) if int(e) > self.B else self.B
            out.append(flat[off:off + e ** 3].reshape(e, e, e))
            off += e ** 3
        return out

    @property
    def memory_mode(self) -> str:
        m = int(lib().pfb_sim3d_memory_mode(self._h))
        return {v: k for k, v in self.MEMORY_MODES.items()}[m]

    @property
    def scratch_slots(self) -> int:
        return int(lib().pfb_sim3d_scratch_slots(self._h))

    @property
    def promoted_count(self) -> int:
        return int(lib().pfb_sim3d_promoted_count(self._h))

    @property
    def max_edge(self) -> int:
        return int(lib().pfb_sim3d_max_edge(self._h))

    @property
    def recoveries(self) -> int:
        return int(lib().pfb_sim3d_recoveries(self._h))

    def set_order(self, morton: bool) -> None:
        """Visit cells in the Morton order of their bricks (default) or in
        slot order; results do not depend on it."""
        check(lib().pfb_sim3d_set_order(self._h, 1 if morton else 0), "set_order")

    def measure_current(self) -> None:
        """Measure the current state and set velocities without a tumble (as
        the reference does before output and checkpoints)."""
        check(lib().pfb_sim3d_measure_current(self._h), "measure_current")

    def verify(self) -> tuple[float, int, int]:
        """(max relative volume error, max aggregate word, support voxels on a
        brick face or outside the domain) after measuring the current state."""
        rel, smax, edges = C.c_double(), C.c_uint32(), C.c_ulonglong()
        check(lib().pfb_sim3d_verify(self._h, C.byref(rel), C.byref(smax), C.byref(edges)), "verify")
        return rel.value, smax.value, edges.value

    def measure_wall(self) -> None:
        """Channel wall diagnostics of the current field into the cell
        records (wall_overlap, outside_slit_volume)."""
        check(lib().pfb_sim3d_measure_wall(self._h), "measure_wall")

    def boundary_open(self, path, interval: int, projection: str = "maximum",
                      compress: bool = False) -> None:
        """Start a PFB3D boundary recording in a new file (header only);
        projection "maximum" or "basal" (substrate slab)."""
        proj = {"basal": 1, "maximum": 2}[projection]
        check(lib().pfb_sim3d_boundary_open(self._h, str(path).encode(), proj, interval,
                                            1 if compress else 0), "boundary_open")

    def boundary_capture(self) -> None:
        check(lib().pfb_sim3d_boundary_capture(self._h), "boundary_capture")

    def boundary_close(self, complete: bool = True) -> None:
        check(lib().pfb_sim3d_boundary_close(self._h, 1 if complete else 0), "boundary_close")

    def bench(self, warmup: int, steps: int) -> float:
        ms = C.c_double()
        check(lib().pfb_sim3d_bench(self._h, warmup, steps, C.byref(ms)), "bench")
        return ms.value

    @property
    def step(self) -> int:
        return int(lib().pfb_sim3d_step(self._h))

    @property
    def stream(self) -> int:
        return int(lib().pfb_sim3d_stream(self._h) or 0)

    def cells(self) -> np.ndarray:
        out = np.zeros(self.params.num_cells, CELL3D_DTYPE)
        check(lib().pfb_sim3d_get_cells(self._h, ptr(out)), "get_cells")
        return out

    def phi(self) -> np.ndarray:
        B = self.B
        out = np.zeros((self.params.num_cells, B, B, B), np.float32)
        check(lib().pfb_sim3d_get_phi(self._h, ptr(out)), "get_phi")
        return out

    def S(self) -> np.ndarray:
        L = self.layout
        out = np.zeros((L.nz, L.ny, L.pitch_x), np.uint32)
        check(lib().pfb_sim3d_get_S(self._h, ptr(out)), "get_S")
        return out

    def flags(self) -> np.ndarray:
        out = np.zeros(FLAG3D_COUNT, np.uint32)
        check(lib().pfb_sim3d_get_flags(self._h, ptr(out)), "get_flags")
        return out

    def update_args(self) -> UpdateArgs3D:
        a = UpdateArgs3D()
        check(lib().pfb_sim3d_update_args(self._h, C.byref(a)), "update_args")
        return a

    def measure_args(self) -> MeasureArgs3D:
        a = MeasureArgs3D()
        check(lib().pfb_sim3d_measure_args(self._h, C.byref(a)), "measure_args")
        return a
