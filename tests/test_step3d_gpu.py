"""3D parity on a B200: this library's launchers against the reference's own
launchers (compiled for sm_100a in oracle/_ref) on byte-identical device
buffers, and against the CPU oracle over several steps.

Exact: seeding, the Q5.27 aggregate, the moment-free update (phi_out and
S_out bit for bit, flags), motion from identical records. Within stated
tolerances: the FP64 moment sums (summation order differs from the
reference's one-CTA fold)."""
import ctypes as C

import numpy as np
import pytest

import oracle3d
import pfb200
from helpers3d import DeviceState3D, small_centres, small_params

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not oracle3d.ref_available(), reason="reference build absent")

GEOMS = ["periodic", "slab", "channel"]
MOMENT_RTOL = 1e-12  # V, C, I, surface: FP64 sums in a different order


def pair(geometry, **kw):
    p = small_params(geometry, **kw)
    c = small_centres(p)
    return p, DeviceState3D(p, c, "pfb"), DeviceState3D(p, c, "ref")


def assert_cells_equal_exact(a, b, fields=("origin_x", "origin_y", "origin_z", "pending_shift_x",
                                           "pending_shift_y", "pending_shift_z", "bb_lo_x",
                                           "bb_hi_x", "bb_lo_y", "bb_hi_y", "bb_lo_z", "bb_hi_z",
                                           "phi_max", "flags", "shift_ctr", "tumble_ctr")):
    for f in fields:
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


def assert_moments_close(a, b):
    for f in ("V", "Cx", "Cy", "Cz", "surface"):
        np.testing.assert_allclose(a[f], b[f], rtol=MOMENT_RTOL, err_msg=f)
    # the integral sums terms of both signs (and, in the channel, the wall
    # term): compare on the scale of its largest component
    scale = max(np.max(np.abs(b[f])) for f in ("Ix", "Iy", "Iz")) + 1e-300
    for f in ("Ix", "Iy", "Iz"):
        assert np.max(np.abs(a[f] - b[f])) <= 1e-10 * scale, f


@needs_ref
@pytest.mark.parametrize("geometry", GEOMS)
def test_seeding_scatter_and_first_measurement_match_reference(geometry):
    p, a, b = pair(geometry)
    np.testing.assert_array_equal(a.get_phi(0), b.get_phi(0))
    np.testing.assert_array_equal(a.get_S(0), b.get_S(0))
    ca, cb = a.get_cells(), b.get_cells()
    assert_cells_equal_exact(ca, cb)
    assert_moments_close(ca, cb)
    np.testing.assert_array_equal(a.get_flags(), b.get_flags())


@needs_ref
@pytest.mark.parametrize("geometry", GEOMS)
def test_update_is_bitwise_identical_to_reference(geometry):
    p, a, b = pair(geometry)
    # identical inputs: the reference's measured records in both
    a.clone_from(b)
    ua, ub = a.update_args(), b.update_args()
    a.S[1].zero_()
    b.S[1].zero_()
    a.update(ua)
    b.update(ub)
    np.testing.assert_array_equal(a.get_phi(1), b.get_phi(1))
    np.testing.assert_array_equal(a.get_S(1), b.get_S(1))
    np.testing.assert_array_equal(a.get_flags(), b.get_flags())
    assert_cells_equal_exact(a.get_cells(), b.get_cells())


@needs_ref
@pytest.mark.parametrize("geometry", GEOMS)
@pytest.mark.parametrize("shift", [(1, 0, 0), (-2, 3, 1), (4, -4, -3), (0, 0, 2)])
def test_recentring_update_matches_reference(geometry, shift):
    p, a, b = pair(geometry)
    a.clone_from(b)
    cells = b.get_cells()
    cells["pending_shift_x"], cells["pending_shift_y"], cells["pending_shift_z"] = shift
    # a supported voxel pushed out of the brick raises DESTINATION_CLIP
    for s in (a, b):
        s.cells.copy_(s.torch.from_numpy(cells.view(np.uint8).copy()).to(s.cells.device))
        s.S[1].zero_()
        s.update(s.update_args())
    np.testing.assert_array_equal(a.get_phi(1), b.get_phi(1))
    np.testing.assert_array_equal(a.get_S(1), b.get_S(1))
    np.testing.assert_array_equal(a.get_flags(), b.get_flags())
    assert_cells_equal_exact(a.get_cells(), b.get_cells())


@needs_ref
@pytest.mark.parametrize("geometry", GEOMS)
def test_motion_with_tumbles_matches_reference(geometry):
    p, a, b = pair(geometry, N=12)
    a.clone_from(b)
    for step in (0, 7, 123456789012):
        for s in (a, b):
            s.step.fill_(step)
            m = s.measure_args(tumble=True, p_tumble=0.5)
            s._call("apply_cell_motion", m)
        ca, cb = a.get_cells(), b.get_cells()
        for f in ("polarity_x", "polarity_y", "polarity_z", "velocity_x", "velocity_y",
                  "velocity_z", "tumble_ctr"):
            np.testing.assert_array_equal(ca[f], cb[f], err_msg=f)
    assert int(cb["tumble_ctr"].sum()) > 0


@needs_ref
@pytest.mark.parametrize("geometry", GEOMS)
def test_multi_step_tracks_reference(geometry):
    p, a, b = pair(geometry)
    for _ in range(30):
        a.step_once()
        b.step_once()
    assert int(a.step.item()) == int(b.step.item()) == 30
    np.testing.assert_array_equal(a.get_flags(), b.get_flags())
    ca, cb = a.get_cells(), b.get_cells()
    for f in ("origin_x", "origin_y", "origin_z", "shift_ctr", "tumble_ctr", "flags"):
        np.testing.assert_array_equal(ca[f], cb[f], err_msg=f)
    np.testing.assert_allclose(ca["V"], cb["V"], rtol=1e-9)
    assert np.max(np.abs(a.get_phi() - b.get_phi())) <= 1e-6


@pytest.mark.parametrize("geometry", GEOMS)
def test_multi_step_vs_cpu_oracle(geometry):
    p = small_params(geometry)
    c = small_centres(p)
    a = DeviceState3D(p, c, "pfb")
    wall = a.wall.cpu().numpy() if a.wall is not None else None
    o32 = oracle3d.OracleState3D(p, a.layout, a.B, a.get_cells(), a.get_phi(), a.get_S(),
                                 wall=wall)
    for _ in range(20):
        a.step_once()
    assert o32.advance(20) == [0] * 20
    ca = a.get_cells()
    for f in ("origin_x", "origin_y", "origin_z"):
        np.testing.assert_array_equal(ca[f], o32.cells[f], err_msg=f)
    np.testing.assert_allclose(ca["V"], o32.cells["V"], rtol=1e-5)
    assert np.max(np.abs(a.get_phi() - o32.phi)) <= 1e-5
    assert int(a.get_flags().sum()) == 0


@needs_ref
def test_fatal_step_keeps_the_accepted_state():
    p, a, b = pair("periodic")
    a.clone_from(b)
    for s in (a, b):
        phi = s.phi[s.cur]
        phi[2, 10, 11, 12] = float("nan")
    before_cells = a.get_cells()
    before_phi = a.get_phi()
    for s in (a, b):
        s.step_once()
    for s in (a, b):
        fl = s.get_flags()
        assert fl[3] > 0  # NONFINITE
        assert int(s.step.item()) == 0  # not advanced
        after = s.get_cells()
        assert_cells_equal_exact(after, before_cells)
        np.testing.assert_array_equal(np.isnan(s.get_phi()), np.isnan(before_phi))
        np.testing.assert_array_equal(np.nan_to_num(s.get_phi()), np.nan_to_num(before_phi))
    np.testing.assert_array_equal(a.get_S(), b.get_S())


def test_sim3d_driver_runs_and_conserves_volume():
    p = small_params("periodic", N=8)
    sim = pfb200.Sim3D(p, small_centres(p))
    sim.advance(25)
    assert sim.step == 25
    assert int(sim.flags().sum()) == 0
    cells = sim.cells()
    # the diffuse profile relaxes from the calibrated seed within a few percent
    np.testing.assert_allclose(cells["V"], p.volume0, rtol=0.1)
    S = sim.S()
    phi = sim.phi()
    assert S.max() > 0 and np.isfinite(phi).all()
    sim.close()
