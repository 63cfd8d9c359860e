"""The fused 3D step (pfb3d_step_fused: measurement, motion and update of a
cell in one cluster launch) on a B200:

* against the reference's own launchers (oracle/_ref/libref3d.so) at the
  benchmarked configurations (periodic 256^3 with 512 cells and the slab
  256 x 256 x 128 with 187 cells, lambda 7, R 10, B 64) and at B 40 in all
  three geometries: the committed measurement
  equals the reference's to 1e-12, and the reference's update run on the
  fused kernel's committed records gives bit-identical phi, S and flags.
  Bricks are moved inside their windows before a step so that the fused
  kernel plans recentring shifts itself (z shifts restage the planes);
* the driver's fused path against its separate launches over many steps:
  cells, phi, S and flags bit-identical (same moment grouping), with and
  without the CUDA graph;
* the visit order of the cells (Morton or slot order) changes no result;
* a fatal step (a planted NaN): after the repair and restore both paths
  leave the same phi, S, cells and flags as the reference.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle3d
import pfb200
from helpers3d import DeviceState3D, small_centres, small_params
from test_bench_config_parity_gpu import assert_measure_3d, c3_centres, c3_params, set_cells

pytestmark = pytest.mark.gpu
needs_ref3 = pytest.mark.skipif(not oracle3d.ref_available(), reason="reference 3D build absent")


def finish_step(s: DeviceState3D, u) -> None:
    """Repair, origin finalisation, restore and step counter (the Sim3D
    sequence after the update), then the buffer flip."""
    s._call("repair_after_fatal", u)
    s._call("finalize_origins", s.cells.data_ptr(), s.N, s.flags.data_ptr())
    s._call("restore_cells_after_fatal", s.cells.data_ptr(), s.accepted.data_ptr(), s.N,
            s.flags.data_ptr(), *([None] if s.impl == "pfb" else []))
    s._call("advance_step", s.step.data_ptr(), s.flags.data_ptr())
    s.cur = 1 - s.cur
    s.steps_done += 1
    torch.cuda.synchronize()


def fused_launch(s: DeviceState3D, surface: bool):
    s.accepted.copy_(s.cells)
    m = s.measure_args(tumble=True, surface=surface)
    s.S[1 - s.cur].zero_()
    u = s.update_args()
    rc = pfb200.lib().pfb3d_step_fused(C.byref(m), C.byref(u), None)
    assert rc == 0, pfb200.lib().pfb_last_error()
    torch.cuda.synchronize()
    return u


def device_status() -> int:
    st = C.c_uint(0)
    assert pfb200.lib().pfb3d_device_status(C.byref(st), 1) == 0
    return st.value


def move_bricks(s: DeviceState3D, with_z: bool, seed: int) -> None:
    """Move each brick's field by d (|d| <= 2 per axis, keeping the support
    at least one voxel from the brick faces) inside its window and its origin
    by -d: the world field and S are unchanged, the centroid leaves the brick
    centre by about d."""
    rng = np.random.default_rng(seed)
    cells = s.get_cells()
    phi = s.phi[s.cur]
    B = s.B
    for n in range(s.N):
        mask = phi[n].abs() > 1e-5
        d = np.zeros(3, int)
        for axis, dims in ((0, (0, 1)), (1, (0, 2)), (2, (1, 2))):  # x, y, z of phi[z, y, x]
            if axis == 2 and not with_z:
                continue
            idx = torch.nonzero(mask.any(dim=dims)).flatten()
            lo, hi = int(idx.min()), int(idx.max())
            d[axis] = int(rng.integers(max(-2, 1 - lo), min(2, B - 2 - hi) + 1))
        phi[n] = torch.roll(phi[n], shifts=(int(d[2]), int(d[1]), int(d[0])), dims=(0, 1, 2))
        cells["origin_x"][n] -= d[0]
        cells["origin_y"][n] -= d[1]
        cells["origin_z"][n] -= d[2]
    set_cells(s, cells)
    torch.cuda.synchronize()


def fused_vs_reference(p, centres, steps=3, move_at=1):
    b = DeviceState3D(p, centres, "ref")
    a = DeviceState3D(p, centres, "pfb")
    K = pfb200.lib().pfb3d_step_cluster(a.B)
    assert K > 0
    planned = 0
    for k in range(steps):
        if k == move_at:
            move_bricks(b, p.geometry == "periodic", seed=7 + k)
        a.clone_from(b)
        u_a = fused_launch(a, surface=(k == 0))
        # the reference measures the same state
        b.accepted.copy_(b.cells)
        m = b.measure_args(tumble=True, surface=(k == 0))
        b._call("measure_cells_only", m)
        b._call("apply_cell_motion", m)
        ca, cb = a.get_cells(), b.get_cells()
        assert_measure_3d(ca, cb, B=a.B)
        for f in ("velocity_x", "velocity_y", "velocity_z", "polarity_x", "polarity_y",
                  "polarity_z"):
            np.testing.assert_allclose(ca[f], cb[f], rtol=1e-6, atol=1e-12, err_msg=f)
        planned += int(np.count_nonzero(ca["pending_shift_x"] | ca["pending_shift_y"]
                                        | ca["pending_shift_z"]))
        if k == move_at:
            assert np.count_nonzero(ca["pending_shift_x"] | ca["pending_shift_y"]) >= p.num_cells // 3
            if p.geometry == "periodic":
                assert np.count_nonzero(ca["pending_shift_z"]) >= p.num_cells // 5
        # the reference's update on the fused kernel's committed records
        set_cells(b, ca)
        b.S[1 - b.cur].zero_()
        u_b = b.update_args()
        b.update(u_b)
        torch.cuda.synchronize()
        assert np.array_equal(a.get_phi(1 - a.cur), b.get_phi(1 - b.cur)), f"phi differs, step {k}"
        np.testing.assert_array_equal(a.get_S(1 - a.cur), b.get_S(1 - b.cur))
        np.testing.assert_array_equal(a.get_flags(), b.get_flags())
        finish_step(a, u_a)
        finish_step(b, u_b)
        ca, cb = a.get_cells(), b.get_cells()
        for f in ("origin_x", "origin_y", "origin_z", "shift_ctr", "tumble_ctr", "flags"):
            np.testing.assert_array_equal(ca[f], cb[f], err_msg=f)
    assert planned >= p.num_cells // 3
    assert int(a.get_flags().sum()) == 0
    assert device_status() == 0


@needs_ref3
def test_fused_c3_periodic_256_against_reference():
    p = c3_params("periodic", 512, 256, 256)
    assert pfb200.lib().pfb3d_step_cluster(64) == 4
    fused_vs_reference(p, c3_centres(p))


@needs_ref3
def test_fused_c3_slab_256x256x128_against_reference():
    p = c3_params("slab", 187, 256, 128)
    fused_vs_reference(p, c3_centres(p))


@needs_ref3
@pytest.mark.parametrize("geometry", ["periodic", "slab", "channel"])
def test_fused_small_bricks_against_reference(geometry):
    p = small_params(geometry)
    assert pfb200.lib().pfb3d_step_cluster(p.brick()) == 4
    fused_vs_reference(p, small_centres(p), steps=4)


def run_driver(p, centres, steps, fused, graph=True, morton=True):
    s = pfb200.Sim3D(p, centres)
    assert not s.fused  # the separate launches are the default
    s.set_fused(fused)
    s.set_graph(graph)
    if not morton:
        s.set_order(False)
    assert s.fused == fused
    s.advance(steps)
    out = (s.cells(), s.phi(), s.S(), s.flags())
    s.close()
    return out


def assert_same_state(x, y):
    assert x[0].tobytes() == y[0].tobytes()
    assert x[1].tobytes() == y[1].tobytes()
    assert x[2].tobytes() == y[2].tobytes()
    np.testing.assert_array_equal(x[3], y[3])


@pytest.mark.parametrize("geometry", ["periodic", "slab", "channel"])
def test_driver_fused_equals_separate_launches(geometry):
    p = small_params(geometry, full_moment_every=5)
    c = small_centres(p)
    a = run_driver(p, c, 23, fused=True)
    b = run_driver(p, c, 23, fused=False)
    assert_same_state(a, b)
    g = run_driver(p, c, 23, fused=True, graph=False)
    assert_same_state(a, g)
    assert device_status() == 0


def test_driver_fused_equals_separate_launches_b64():
    p = pfb200.SimParams3D(Nx=128, Ny=128, Nz=128, geometry="periodic", num_cells=64,
                           target_radius=10.0, lambda_=7.0, B=64, seed=1234, full_moment_every=10)
    c = pfb200.sequential_centres(64, 128, 20.0, 1234, first_at_centre=True)
    a = run_driver(p, c, 40, fused=True)
    b = run_driver(p, c, 40, fused=False)
    assert_same_state(a, b)
    assert not a[3].any()


@pytest.mark.parametrize("fused", [True, False])
def test_driver_visit_order_changes_nothing(fused):
    p = pfb200.SimParams3D(Nx=128, Ny=128, Nz=128, geometry="periodic", num_cells=64,
                           target_radius=10.0, lambda_=7.0, B=64, seed=99, full_moment_every=7)
    c = pfb200.sequential_centres(64, 128, 20.0, 99)
    a = run_driver(p, c, 16, fused=fused)
    b = run_driver(p, c, 16, fused=fused, morton=False)
    assert_same_state(a, b)


@needs_ref3
def test_fused_fatal_step_rolls_back_like_reference():
    p = small_params("periodic")
    c = small_centres(p)
    ref = DeviceState3D(p, c, "ref")
    mine = DeviceState3D(p, c, "pfb")
    mine.clone_from(ref)
    states = {}
    for s in (mine, ref):
        s.phi[s.cur][2, 20, 21, 19] = float("nan")
        torch.cuda.synchronize()
        if s.impl == "pfb":
            u = fused_launch(s, surface=False)
        else:
            s.accepted.copy_(s.cells)
            m = s.measure_args(tumble=True, surface=False)
            s._call("measure_cells_only", m)
            s._call("apply_cell_motion", m)
            s.S[1 - s.cur].zero_()
            u = s.update_args()
            s.update(u)
        finish_step(s, u)
        states[s.impl] = (s.get_cells(), s.get_phi(), s.get_S(), s.get_flags(), s.step.item())
    a, b = states["pfb"], states["ref"]
    assert a[0].tobytes() == b[0].tobytes()
    np.testing.assert_array_equal(np.nan_to_num(a[1], nan=7.0), np.nan_to_num(b[1], nan=7.0))
    np.testing.assert_array_equal(a[2], b[2])
    np.testing.assert_array_equal(a[3], b[3])
    assert a[3][pfb200.FLAG3D_NAMES.index("nonfinite")] > 0
    assert a[4] == b[4] == 0
