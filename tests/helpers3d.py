"""Test fixtures of the 3D path: caller-owned device buffers of one 3D system
(torch tensors) in the reference Sim3D's throughput scheme (two phi pools,
two aggregate slots; reference src/pf3d/sim.cu:1460-1651), with the step
sequence driven either through this library's launchers or through the
reference's own (oracle/_ref/libref3d.so) on the same buffers."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

import oracle3d
import pfb200
from pfb200 import CELL3D_DTYPE
from pfb200._abi3d import (BOUNDARY_HARD_WALL_CHANNEL, InitArgs3D, Layout3D, MeasureArgs3D,
                           ScatterArgs3D, UpdateArgs3D, Vec3)
from pfb200.sim3d import GEOMETRIES, SimParams3D


def wall_profile(p: SimParams3D) -> np.ndarray:
    """kappa_w/kappa psi_w^2 per plane (reference src/pf3d/sim.cu:647-664)."""
    ratio = np.float32(p.wall_kappa / p.kappa)
    k = 2.7386127875258306 / p.wall_width
    lo, hi = float(p.channel_padding), float(p.channel_padding + p.channel_height)
    out = np.zeros(p.Nz, np.float32)
    for z in range(p.Nz):
        c = z + 0.5
        fluid = 0.25 * (1.0 + math.tanh(k * (c - lo))) * (1.0 - math.tanh(k * (c - hi)))
        w = 1.0 - fluid
        out[z] = ratio * np.float32(w * w)
    return out


def fresh_cells3(p: SimParams3D) -> np.ndarray:
    L = pfb200.lib()
    cells = np.zeros(p.num_cells, CELL3D_DTYPE)
    stream = p.polarity_seed or p.seed
    d = (C.c_double * 3)()
    for i in range(p.num_cells):
        cells[i]["global_id"] = i
        cells[i]["gamma"] = p.gamma
        cells[i]["v_A"] = L.pfb3d_initial_active_speed(i, p.seed, p.v_A, p.v_A_sigma)
        cells[i]["R_tgt"] = p.target_radius
        L.pfb3d_initial_polarity(i, stream, 1 if p.geometry == "slab" else 0, d)
        cells[i]["polarity_x"], cells[i]["polarity_y"], cells[i]["polarity_z"] = d[0], d[1], d[2]
    return cells


class DeviceState3D:
    def __init__(self, p: SimParams3D, centres: np.ndarray, impl: str = "pfb", device="cuda"):
        import torch
        self.torch = torch
        self.p = p
        self.impl = impl
        self.B = p.brick()
        self.N = p.num_cells
        B, N = self.B, self.N
        self.layout = Layout3D(p.Nx, p.Ny, p.Nz, 32 * ((p.Nx + 31) // 32), GEOMETRIES[p.geometry])
        self.s_shape = (p.Nz, p.Ny, self.layout.pitch_x)
        self.phi = [torch.zeros((N, B, B, B), dtype=torch.float32, device=device) for _ in range(2)]
        self.S = [torch.zeros(self.s_shape, dtype=torch.int32, device=device) for _ in range(2)]
        self.cells = torch.from_numpy(fresh_cells3(p).view(np.uint8).copy()).to(device)
        self.accepted = torch.zeros_like(self.cells)
        self.flags = torch.zeros(10, dtype=torch.int32, device=device)
        self.step = torch.zeros(1, dtype=torch.int64, device=device)
        self.cursor = torch.zeros(1, dtype=torch.int64, device=device)
        self.wall = (torch.from_numpy(wall_profile(p)).to(device)
                     if p.geometry == "channel" else None)
        self.cur = 0
        self.steps_done = 0
        self.seed_radius, _ = pfb200.calibrate_seed_radius(p.target_radius, p.lambda_, B)
        c = np.ascontiguousarray(centres, dtype=np.float64).copy()
        if p.geometry == "channel":
            c[:, 2] = (c[:, 2].astype(np.float32) + np.float32(p.channel_padding)
                       - np.float32(0.5)).astype(np.float64)
        self.centres = torch.from_numpy(c).to(device)
        ia = InitArgs3D()
        ia.phi_even = self.phi[0].data_ptr()
        ia.phi_odd = self.phi[1].data_ptr()
        ia.cells = self.cells.data_ptr()
        ia.centres = self.centres.data_ptr()
        ia.N, ia.B = N, B
        ia.layout = self.layout
        ia.lambda_ = p.lambda_
        ia.seed_radius = self.seed_radius
        self._call("initialize_spheres", ia)
        sa = ScatterArgs3D()
        sa.phi, sa.cells, sa.S = self.phi[0].data_ptr(), self.cells.data_ptr(), self.S[0].data_ptr()
        sa.global_flags = self.flags.data_ptr()
        sa.layout = self.layout
        sa.N, sa.B = N, B
        self._call("scatter_current", sa)
        m = self.measure_args(tumble=False, surface=True)
        self._call("measure_cells_only", m)
        self._call("apply_cell_motion", m)
        torch.cuda.synchronize()

    # ---- dispatch ---------------------------------------------------------
    def _call(self, name, *args):
        """Call the 3D launcher `name` of the selected implementation; record
        arguments are passed by address."""
        if self.impl == "pfb":
            conv = [C.byref(a) if isinstance(a, C.Structure) else a for a in args]
            rc = getattr(pfb200.lib(), "pfb3d_" + name)(*conv, None)
            assert rc == 0, pfb200.lib().pfb_last_error()
        else:
            conv = [C.addressof(a) if isinstance(a, C.Structure) else a for a in args]
            rc = getattr(oracle3d.rlib(), "ref3d_" + name)(*conv, None)
            assert rc == 0, name

    def update(self, u):
        if self.impl == "pfb":
            rc = pfb200.lib().pfb3d_update(C.byref(u), None)
            assert rc == 0, pfb200.lib().pfb_last_error()
        elif self.p.geometry == "periodic":
            assert oracle3d.rlib().ref3d_update_periodic(C.addressof(u), None) == 0
        else:
            assert oracle3d.rlib().ref3d_update_tiled(C.addressof(u), 148 * 2, None) == 0

    # ---- argument records -------------------------------------------------
    def measure_args(self, tumble=True, surface=False, p_tumble=None) -> MeasureArgs3D:
        p = self.p
        m = MeasureArgs3D()
        m.phi = self.phi[self.cur].data_ptr()
        m.S = self.S[self.cur].data_ptr()
        if self.wall is not None:
            m.wall.values, m.wall.planes = self.wall.data_ptr(), p.Nz
        m.cells = self.cells.data_ptr()
        m.global_flags = self.flags.data_ptr()
        m.step = self.step.data_ptr()
        m.layout = self.layout
        m.N, m.B = self.N, self.B
        m.shards = 1
        m.polarity_stream = p.polarity_seed or p.seed
        m.aging_steps = int(p.aging_time / p.dt + 0.5)
        m.p_tumble = -math.expm1(-p.dt / p.tau) if p_tumble is None else p_tumble
        m.motility_coeff = 60.0 * p.kappa / (p.lambda_ ** 2) / p.xi
        m.max_shift, m.support_margin = 4, 8
        m.apply_tumble, m.compute_surface = int(tumble), int(surface)
        return m

    def update_args(self) -> UpdateArgs3D:
        p = self.p
        u = UpdateArgs3D()
        u.phi_in, u.phi_out = self.phi[self.cur].data_ptr(), self.phi[1 - self.cur].data_ptr()
        u.S_in, u.S_out = self.S[self.cur].data_ptr(), self.S[1 - self.cur].data_ptr()
        if self.wall is not None:
            u.wall.values, u.wall.planes = self.wall.data_ptr(), p.Nz
        u.cells = self.cells.data_ptr()
        u.global_flags = self.flags.data_ptr()
        u.work_cursor = self.cursor.data_ptr()
        u.layout = self.layout
        u.N, u.B = self.N, self.B
        u.dt = p.dt
        u.V0 = p.volume0
        u.volume_scale = 2.0 * p.mu / p.volume0
        u.bulk_scale = 30.0 / p.lambda_ ** 2
        u.interaction_coeff = 60.0 * p.kappa / p.lambda_ ** 2
        return u

    # ---- one step of the Sim3D sequence -----------------------------------
    def step_once(self, p_tumble=None):
        torch = self.torch
        full = self.p.full_moment_every > 0 and self.steps_done % self.p.full_moment_every == 0
        self.accepted.copy_(self.cells)
        m = self.measure_args(tumble=True, surface=full, p_tumble=p_tumble)
        self._call("measure_cells_only", m)
        self._call("apply_cell_motion", m)
        self.S[1 - self.cur].zero_()
        u = self.update_args()
        self.update(u)
        self._call("repair_after_fatal", u)
        self._call("finalize_origins", self.cells.data_ptr(), self.N, self.flags.data_ptr())
        self._call("restore_cells_after_fatal", self.cells.data_ptr(), self.accepted.data_ptr(),
                   self.N, self.flags.data_ptr(), *([None] if self.impl == "pfb" else []))
        self._call("advance_step", self.step.data_ptr(), self.flags.data_ptr())
        self.cur = 1 - self.cur
        self.steps_done += 1
        torch.cuda.synchronize()

    # ---- host views ---------------------------------------------------------
    def get_cells(self):
        self.torch.cuda.synchronize()
        return self.cells.cpu().numpy().view(CELL3D_DTYPE).copy()

    def get_phi(self, which=None):
        return self.phi[self.cur if which is None else which].cpu().numpy()

    def get_S(self, which=None):
        return self.S[self.cur if which is None else which].cpu().numpy().view(np.uint32)

    def get_flags(self):
        return self.flags.cpu().numpy().view(np.uint32).copy()

    def clone_from(self, other: "DeviceState3D"):
        """Copy every buffer of `other` (same shapes) into this state."""
        for a, b in zip(self.phi, other.phi):
            a.copy_(b)
        for a, b in zip(self.S, other.S):
            a.copy_(b)
        self.cells.copy_(other.cells)
        self.flags.copy_(other.flags)
        self.step.copy_(other.step)
        self.cur, self.steps_done = other.cur, other.steps_done
        self.torch.cuda.synchronize()


def small_params(geometry="periodic", N=6, **kw) -> SimParams3D:
    """R = 4, lambda = 3 cells in B = 40 bricks (8 voxels of margin over the
    automatic edge) on small domains."""
    base = dict(num_cells=N, lambda_=3.0, target_radius=4.0, B=40, v_A=0.05, seed=42)
    if geometry == "periodic":
        base.update(Nx=80, Ny=80, Nz=80)
    elif geometry == "slab":
        base.update(Nx=80, Ny=80, Nz=56, geometry="slab")
    else:
        base.update(Nx=80, Ny=80, Nz=30, geometry="channel", channel_height=24,
                    channel_padding=3, wall_kappa=5.0, wall_width=1.0)
    base.update(kw)
    return SimParams3D(**base)


def small_centres(p: SimParams3D, seed=3) -> np.ndarray:
    if p.geometry == "periodic":
        return pfb200.sequential_centres(p.num_cells, p.Nx, 2 * p.target_radius, seed)
    if p.geometry == "slab":
        return pfb200.sequential_centres(p.num_cells, p.Nx, 2 * p.target_radius, seed,
                                         planar_z=-0.5)
    return pfb200.sequential_centres(p.num_cells, p.Nx, 2 * p.target_radius, seed,
                                     height=p.channel_height, z_margin=p.target_radius + 1)
