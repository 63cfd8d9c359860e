"""Shared test fixtures for the 2D path: parameter sets, a synthetic state
that exercises every shape class, device buffers held in torch tensors, and
world-frame comparisons."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

import pfb200
from pfb200 import CELL_DTYPE, CLASSES, SimParams2D, StepArgs2D


def params(L: int, N: int, R: float = 12.0, **kw) -> SimParams2D:
    p = SimParams2D(L=L, num_cells=N, target_radius=R)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def fresh_cells(p: SimParams2D) -> np.ndarray:
    """Per-cell records of a fresh start (reference src/sim.cu:136-145, 324-340)."""
    L = pfb200.lib()
    N = p.num_cells
    cells = np.zeros(N, CELL_DTYPE)
    n_cancer = int(round(p.cancer_fraction * N))
    pstream = p.polarity_seed or p.seed
    for i in range(N):
        cells[i]["global_id"] = i
        cells[i]["gamma"] = p.gamma_cancer if i < n_cancer else p.gamma_normal
        cells[i]["v_A"] = L.pfb_ic_v_A(i, p.seed, p.v_A, p.v_A_sigma)
        cells[i]["M_pf"] = p.phase_field_mobility
        cells[i]["R_tgt"] = p.target_radius
        cells[i]["theta"] = L.pfb_ic_theta(i, pstream)
    return cells


def synthetic_all_classes(L: int = 701, seed: int = 7):
    """Six cells, one per shape class, with asymmetric bumps, periodic wrap,
    forced promotion/demotion on a few cells and non-trivial recentring."""
    rng = np.random.default_rng(seed)
    N = 6
    cells = np.zeros(N, CELL_DTYPE)
    phi = np.zeros((N, 288, 288), np.float32)
    centres = [(L - 30, 40), (200, L - 20), (350, 350), (520, 150), (100, 500), (600, 600)]
    for i in range(N):
        wx, wy, tx0, ty0 = CLASSES[i]
        c = cells[i]
        c["global_id"] = 11 + 17 * i
        c["cls"] = i
        c["cls_written"] = (i, i)
        c["gamma"] = 1.0 if i % 2 == 0 else 0.35
        c["M_pf"] = 0.5 if i < 4 else 0.3
        c["v_A"] = 0.01
        c["R_tgt"] = 12.0
        c["theta"] = 0.3 + i
        cx, cy = centres[i]
        c["gx0"] = (cx - wx // 2) % L
        c["gy0"] = (cy - wy // 2) % L
        y, x = np.mgrid[0:wy, 0:wx].astype(np.float64)
        sx, sy = 0.16 * wx, 0.13 * wy
        X = (x - 0.5 * wx - 2.5) / sx
        Y = (y - 0.5 * wy + 1.5) / sy
        z = 0.8 * np.exp(-0.5 * (X * X + Y * Y)) * (1.0 + 0.07 * X * Y + 0.05 * X)
        z += 1e-4 * rng.standard_normal(z.shape)
        z = np.clip(z, 0.0, None)
        phi[i, ty0:ty0 + wy, tx0:tx0 + wx] = z.astype(np.float32)
    # moments of the stored field, as k_init_moments would leave them
    for i in range(N):
        wx, wy, tx0, ty0 = CLASSES[i]
        w = phi[i, ty0:ty0 + wy, tx0:tx0 + wx].astype(np.float64)
        d = w * w
        yy, xx = np.mgrid[0:wy, 0:wx]
        cells[i]["V"] = d.sum()
        cells[i]["Cx"] = (d * xx).sum()
        cells[i]["Cy"] = (d * yy).sum()
        sup = np.argwhere(w > 1e-5)
        cells[i]["bb_lo_y"], cells[i]["bb_lo_x"] = sup.min(0)
        cells[i]["bb_hi_y"], cells[i]["bb_hi_x"] = sup.max(0)
        cells[i]["phi_max"] = np.abs(w).max()
    # cell 0: support extent forcing promotion out of class 0
    cells[0]["bb_lo_x"], cells[0]["bb_hi_x"] = 2, 139
    # cell 3 (160^2): small support with the dwell about to expire -> demotion
    cells[3]["bb_lo_x"], cells[3]["bb_hi_x"] = 50, 90
    cells[3]["bb_lo_y"], cells[3]["bb_hi_y"] = 50, 90
    cells[3]["promote_ctr"] = 199
    # cell 1: centroid offset -> clamped shift of 4
    cells[1]["Cx"] += 9.0 * cells[1]["V"]
    return cells, phi


class DeviceState2D:
    """Caller-owned device buffers of one 2D system (torch tensors), in the
    slot scheme of the reference host driver (src/sim.cu:578-618)."""

    def __init__(self, p: SimParams2D, cells: np.ndarray, phi: np.ndarray, step: int = 0,
                 device: str = "cuda"):
        import torch
        self.torch = torch
        self.p = p
        self.N = p.num_cells
        self.L = p.L
        self.P = 32 * ((p.L + 31) // 32)
        self.step = step
        pin = step % 2
        pool = np.ascontiguousarray(phi, dtype=np.float32).reshape(self.N, 288, 288)
        self.phi = [torch.zeros((self.N, 288, 288), dtype=torch.float32, device=device)
                    for _ in range(2)]
        self.phi[pin].copy_(torch.from_numpy(pool))
        self.S = torch.zeros((3, self.L, self.P), dtype=torch.int32, device=device)
        c = np.ascontiguousarray(cells.copy())
        c["cls_written"][:, 0] = c["cls"]
        c["cls_written"][:, 1] = c["cls"]
        self.cells = torch.from_numpy(c.view(np.uint8).copy()).to(device)
        self.cls = torch.from_numpy(np.ascontiguousarray(c["cls"]).astype(np.uint8)).to(device)
        self.cursor = torch.zeros(2, dtype=torch.int64, device=device)
        st = np.array([step if pin == 0 else step + 1, step if pin == 1 else step + 1], np.int64)
        self.steps = torch.from_numpy(st).to(device)
        self.flags = torch.zeros(8, dtype=torch.int32, device=device)
        # identity visit order: the reference kernel dereferences perm
        self.perm = torch.arange(self.N, dtype=torch.int32, device=device)
        # S^step from the pool
        rc = pfb200.lib().pfb_scatter_all2d(
            self.phi[pin].data_ptr(), self.cells.data_ptr(), self.cls.data_ptr(),
            self.S[step % 3].data_ptr(), self.N, self.L, self.P, self.flags.data_ptr(), None)
        pfb200.check(rc, "scatter_all")
        torch.cuda.synchronize()
        self.coeff = pfb200.step_coefficients(p)

    def args(self) -> StepArgs2D:
        slot = self.step
        pin, pout, rs = slot % 2, 1 - slot % 2, slot % 3
        a = StepArgs2D()
        C.memmove(C.byref(a), C.byref(self.coeff), C.sizeof(StepArgs2D))
        a.phi_in = self.phi[pin].data_ptr()
        a.phi_out = self.phi[pout].data_ptr()
        a.S_rd = self.S[rs].data_ptr()
        a.S_sc = self.S[(rs + 1) % 3].data_ptr()
        a.S_cl = self.S[(rs + 2) % 3].data_ptr()
        a.cell = self.cells.data_ptr()
        a.cell_cls = self.cls.data_ptr()
        a.perm = self.perm.data_ptr()
        a.cursor_use = self.cursor.data_ptr() + 8 * pin
        a.cursor_clear = self.cursor.data_ptr() + 8 * pout
        a.step_rd = self.steps.data_ptr() + 8 * pin
        a.step_wr = self.steps.data_ptr() + 8 * pout
        a.flags = self.flags.data_ptr()
        a.moments = None
        a.N, a.L, a.P, a.parity_out = self.N, self.L, self.P, pout
        a.clear_ahead_words = self.L * self.P
        return a

    def step_with(self, launch) -> None:
        """launch(args) issues one step on the legacy stream; advances slot."""
        rc = launch(self.args())
        assert rc == 0, pfb200.lib().pfb_last_error()
        self.step += 1

    def sync(self):
        self.torch.cuda.synchronize()

    def get_cells(self) -> np.ndarray:
        self.sync()
        return self.cells.cpu().numpy().view(CELL_DTYPE).copy()

    def get_phi(self) -> np.ndarray:
        self.sync()
        return self.phi[self.step % 2].cpu().numpy()

    def get_S(self) -> np.ndarray:
        self.sync()
        return self.S[self.step % 3].cpu().numpy().view(np.uint32)

    def get_flags(self) -> np.ndarray:
        self.sync()
        return self.flags.cpu().numpy().view(np.uint32)


def world_fields(phi: np.ndarray, cells: np.ndarray, L: int) -> np.ndarray:
    """(N, L, L) per-cell fields on the periodic lattice (world frame)."""
    out = np.zeros((len(cells), L, L), np.float64)
    for n in range(len(cells)):
        out[n] = pfb200.world_field(phi, cells, n, L)
    return out


def max_world_diff(phi_a, cells_a, phi_b, cells_b, L) -> float:
    worst = 0.0
    for n in range(len(cells_a)):
        a = pfb200.world_field(phi_a, cells_a, n, L)
        b = pfb200.world_field(phi_b, cells_b, n, L)
        worst = max(worst, float(np.abs(a - b).max()))
    return worst


def s_from_phi(phi: np.ndarray, cells: np.ndarray, L: int) -> np.ndarray:
    """Exact Q5.27 aggregate of a stored pool (integer sums)."""
    import oracle2d
    P = 32 * ((L + 31) // 32)
    S, _ = oracle2d.scatter_all(np.ascontiguousarray(phi, np.float32),
                                np.ascontiguousarray(cells), L, P)
    return S


def pair_sep(cx, cy, L) -> float:
    best = math.inf
    for i in range(len(cx)):
        for j in range(i):
            dx = (cx[i] - cx[j] + L / 2) % L - L / 2
            dy = (cy[i] - cy[j] + L / 2) % L - L / 2
            best = min(best, math.hypot(dx, dy))
    return best
