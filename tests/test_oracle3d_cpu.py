"""Pins of the 3D oracle and of the library's 3D host helpers against the
reference's own host code, compiled in place from the reference sources
(oracle/_ref/libref3d_cpu.so: include/pf3d/reference.hpp and
include/pf3d/rng.cuh):

* the seed-radius calibration (reference.hpp:712-745) bit for bit;
* the Philox draws of initial polarity, active speed and tumbles
  (rng.cuh:41-150) bit for bit;
* one FP64 step of the oracle against the reference's dense FP64 one-step
  (reference.hpp:219-292) on two overlapping cells of a periodic box.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle3d
import pfb200
from pfb200 import CELL3D_DTYPE, Layout3D, SimParams3D

needs_ref = pytest.mark.skipif(not oracle3d.ref_cpu_available(), reason="reference build absent")


@needs_ref
@pytest.mark.parametrize("R,lam,B", [(10.0, 7.0, 64), (4.0, 3.0, 32), (12.0, 7.0, 72)])
def test_calibration_matches_reference(R, lam, B):
    s, v = pfb200.calibrate_seed_radius(R, lam, B)
    rs, rv = C.c_double(), C.c_double()
    assert oracle3d.rclib().ref3d_cpu_calibrate(R, lam, B, C.byref(rs), C.byref(rv)) == 0
    assert s == rs.value and v == rv.value


def test_automatic_brick_edge_matches_reference_cli():
    # the reference CLI prints B=64 for R=10, lambda=7 ("minimum aligned B=64")
    assert pfb200.automatic_brick_edge(10.0, 7.0) == 64
    assert pfb200.automatic_brick_edge(4.0, 3.0) == 32


@needs_ref
def test_philox_draws_match_reference():
    L = pfb200.lib()
    R = oracle3d.rclib()
    a = (C.c_double * 3)()
    b = (C.c_double * 3)()
    for stream in (0, 1234, 0xDEADBEEFCAFE):
        for gid in list(range(40)) + [2**33 + 7]:
            for planar in (0, 1):
                L.pfb3d_initial_polarity(gid, stream, planar, a)
                R.ref3d_cpu_initial_polarity(gid, stream, planar, b)
                assert list(a) == list(b)
            assert (L.pfb3d_initial_active_speed(gid, stream, 0.01, 0.3)
                    == R.ref3d_cpu_initial_speed(gid, stream, 0.01, 0.3))
    events = 0
    for step in range(200):
        for gid in (0, 5, 99):
            for planar in (0, 1):
                e1 = L.pfb3d_tumble(step, gid, 77, 0.3, planar, a)
                e2 = R.ref3d_cpu_tumble(step, gid, 77, 0.3, planar, b)
                assert e1 == e2
                if e1:
                    events += 1
                    assert list(a) == list(b)
    assert events > 50


def _brick_sphere(B, centre, seed_r, lam):
    k = math.sqrt(7.5) / lam
    z, y, x = np.meshgrid(np.arange(B), np.arange(B), np.arange(B), indexing="ij")
    r = np.sqrt((x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2)
    return 0.5 * (1.0 - np.tanh(k * (r - seed_r)))


@needs_ref
def test_oracle_f64_step_matches_reference_dense_one_step():
    side, B, lam, R = 48, 32, 3.0, 4.0
    seed_r, _ = pfb200.calibrate_seed_radius(R, lam, B)
    # two overlapping cells; centres within 0.4 of the brick middle so that no
    # recentring shift is planned
    origins = [(3, 5, 2), (12, 9, 10)]
    offsets = [(15.3, 15.6, 15.2), (15.7, 15.4, 15.5)]
    pol = [(1.0, 0.0, 0.0), (0.0, 0.0, -1.0)]
    N = 2
    phi = np.zeros((N, B, B, B))
    cells = np.zeros(N, CELL3D_DTYPE)
    dense = np.zeros((N, side, side, side))
    for n in range(N):
        phi[n] = _brick_sphere(B, offsets[n], seed_r, lam)
        ox, oy, oz = origins[n]
        cells[n]["origin_x"], cells[n]["origin_y"], cells[n]["origin_z"] = ox, oy, oz
        cells[n]["global_id"] = n
        cells[n]["gamma"] = 1.0
        cells[n]["v_A"] = 0.5
        cells[n]["polarity_x"], cells[n]["polarity_y"], cells[n]["polarity_z"] = pol[n]
        dense[n][oz:oz + B, oy:oy + B, ox:ox + B] = phi[n]
    lay = Layout3D(side, side, side, 64, pfb200._abi3d.BOUNDARY_PERIODIC_XYZ)
    # S from the fields (f64 quantisation)
    S = np.zeros((side, side, 64), np.uint32)
    fl = np.zeros(10, np.uint32)
    oracle3d.olib().oracle3d_scatter(1, phi.ctypes.data, cells.ctypes.data, S.ctypes.data,
                                     fl.ctypes.data, C.byref(lay), N, B)
    p = SimParams3D(Nx=side, Ny=side, Nz=side, num_cells=N, B=B, lambda_=lam, target_radius=R,
                    dt=0.01, kappa=10.0, mu=1.0, xi=1500.0, tau=1e300, seed=9)
    st = oracle3d.OracleState3D(p, lay, B, cells, phi, S, f64=True)
    assert st.advance(1) == [0]
    assert int(st.flags.sum()) == 0
    assert (st.cells["pending_shift_x"] == 0).all() and (st.cells["origin_x"] == [3, 12]).all()

    out = np.zeros_like(dense)
    vol = np.zeros(N)
    integ = np.zeros(3 * N)
    vel = np.zeros(3 * N)
    # keep the argument arrays alive across the call
    gamma, speed, polv = np.ones(N), np.full(N, 0.5), np.array(pol, float).ravel()
    rc = oracle3d.rclib().ref3d_cpu_one_step(
        side, N, dense.ctypes.data, gamma.ctypes.data, speed.ctypes.data, polv.ctypes.data,
        0.01, lam, R, 10.0, 1.0, 1500.0, out.ctypes.data, vol.ctypes.data, integ.ctypes.data,
        vel.ctypes.data)
    assert rc == 0
    # the oracle measured the same volume and interaction integral
    np.testing.assert_allclose(st.cells["V"], vol, rtol=1e-13)
    ours_I = np.stack([st.cells["Ix"], st.cells["Iy"], st.cells["Iz"]], 1).ravel()
    np.testing.assert_allclose(ours_I, integ, rtol=1e-11, atol=1e-14)
    for n in range(N):
        ox, oy, oz = origins[n]
        ref_brick = out[n][oz:oz + B, oy:oy + B, ox:ox + B]
        assert np.max(np.abs(st.phi[n] - ref_brick)) <= 1e-13


@needs_ref
def test_oracle_f32_tracks_f64():
    side, B, lam, R = 48, 32, 3.0, 4.0
    seed_r, _ = pfb200.calibrate_seed_radius(R, lam, B)
    N = 2
    phi = np.stack([_brick_sphere(B, (15.4, 15.5, 15.6), seed_r, lam)] * N)
    cells = np.zeros(N, CELL3D_DTYPE)
    cells["origin_x"] = [0, 9]
    cells["origin_y"] = [0, 7]
    cells["origin_z"] = [0, 5]
    cells["global_id"] = [0, 1]
    cells["gamma"] = 1.0
    cells["v_A"] = 0.01
    cells["polarity_x"] = 1.0
    lay = Layout3D(side, side, side, 64, pfb200._abi3d.BOUNDARY_PERIODIC_XYZ)
    S = np.zeros((side, side, 64), np.uint32)
    phi32, fl = phi.astype(np.float32), np.zeros(10, np.uint32)
    oracle3d.olib().oracle3d_scatter(0, phi32.ctypes.data, cells.ctypes.data, S.ctypes.data,
                                     fl.ctypes.data, C.byref(lay), N, B)
    S64 = np.zeros_like(S)
    oracle3d.olib().oracle3d_scatter(1, phi.ctypes.data, cells.ctypes.data, S64.ctypes.data,
                                     fl.ctypes.data, C.byref(lay), N, B)
    p = SimParams3D(Nx=side, Ny=side, Nz=side, num_cells=N, B=B, lambda_=lam, target_radius=R)
    a = oracle3d.OracleState3D(p, lay, B, cells, phi32, S, f64=False)
    b = oracle3d.OracleState3D(p, lay, B, cells, phi, S64, f64=True)
    assert a.advance(20) == [0] * 20
    assert b.advance(20) == [0] * 20
    assert (a.cells["origin_x"] == b.cells["origin_x"]).all()
    assert np.max(np.abs(a.phi - b.phi)) < 2e-5
    np.testing.assert_allclose(a.cells["V"], b.cells["V"], rtol=1e-5)
