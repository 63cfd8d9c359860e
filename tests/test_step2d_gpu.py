"""GPU parity of the sm_100a 2D step (through the C ABI) against

* the CPU oracle (oracle/pf2d_oracle.cpp, binary32 field arithmetic with
  binary64 reductions, every operation separately rounded), and
* the reference's own step kernel compiled in place for sm_100a
  (oracle/_ref/libref2d.so), on byte-identical inputs.

Tolerances (stated here, used below):
  one step          max |dphi| <= 2e-6   (the reference's own GPU-vs-FP64
                                          Euler bound, tests/velocity_observer_test.cu:292-294)
  1000 steps        max |dphi| <= 1e-5   in the world frame
  V, Cx, Cy         relative 1e-7 against the oracle (the GPU contracts
                    multiply-adds, the oracle rounds every operation),
                    1e-9 between GPU builds (binary64 sums in another order)
  velocity          relative 1e-5 + 1e-9 absolute
Integer observables are exact: the Q5.27 aggregate given the stored phi,
tumble counters, classes, origins, support boxes, flags.
"""
import ctypes as C

import numpy as np
import pytest

import oracle2d
import pfb200
from helpers2d import (DeviceState2D, fresh_cells, max_world_diff, params, s_from_phi,
                       synthetic_all_classes)

pytestmark = pytest.mark.gpu

PHI_TOL_1 = 2e-6
PHI_TOL_1000 = 1e-5


def launch_pfb(cluster, variant=0):
    def f(a):
        return pfb200.lib().pfb_step2d_launch_ex(C.byref(a), cluster, variant, None)
    return f


# (cluster size, kernel variant): one cluster of 2, 4 or 8 CTAs per cell
KERNELS = [(2, 1), (4, 1), (8, 1)]


def launch_ref(a):
    return oracle2d.rlib().ref2d_launch_step(C.byref(a), oracle2d.rlib().ref2d_grid(0), None)


def oracle_step(p, cells, phi, step, n=1, f64=False):
    o = oracle2d.OracleSim(p.to_c(), cells, phi, step=step, f64=f64)
    o.advance(n)
    return o


def assert_cells_match(a, b, vel_rtol=1e-5, moment_rtol=1e-7):
    for k in ("gx0", "gy0", "cls", "bb_lo_x", "bb_hi_x", "bb_lo_y", "bb_hi_y", "promote_ctr",
              "shift_ctr", "tumble_ctr", "global_id"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    np.testing.assert_array_equal(a["theta"], b["theta"], err_msg="theta")
    for k in ("V", "Cx", "Cy"):
        np.testing.assert_allclose(a[k], b[k], rtol=moment_rtol, err_msg=k)
    for k in ("vx", "vy"):
        np.testing.assert_allclose(a[k], b[k], rtol=vel_rtol, atol=1e-9, err_msg=k)
    for k in ("Ix", "Iy"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-6, atol=1e-12, err_msg=k)


@pytest.fixture(scope="module", params=[(701, 1), (704, 1), (704, 100), (701, 100)],
                ids=["L701-fm", "L704-fm", "L704", "L701"])
def synth(request):
    # odd and multiple-of-4 sides (the second stages S with bulk copies);
    # full-moment steps every step or not on the tested step
    L, fme = request.param
    cells, phi = synthetic_all_classes(L=L)
    p = params(L, 6, R=12.0, tau=0.02, full_moment_every=fme)  # p_tumble ~ 0.39
    return p, cells, phi


@pytest.mark.parametrize("cluster,variant", KERNELS)
def test_one_step_all_classes_vs_oracle(synth, cluster, variant):
    p, cells, phi = synth
    step = 9000037
    ds = DeviceState2D(p, cells, phi, step=step)
    ds.step_with(launch_pfb(cluster, variant))
    g_cells, g_phi, g_S, g_flags = ds.get_cells(), ds.get_phi(), ds.get_S(), ds.get_flags()
    o = oracle_step(p, cells, phi, step)
    o_cells, o_phi = o.cells(), o.phi()
    # classes 0..5 all took part; some promotion/demotion and tumbles happened
    assert set(cells["cls"]) == set(range(6))
    assert (g_cells["cls"] != cells["cls"]).any()
    assert g_cells["tumble_ctr"].sum() > 0
    assert_cells_match(g_cells, o_cells)
    np.testing.assert_allclose(g_cells["perim"], o_cells["perim"], rtol=1e-6)
    assert max_world_diff(g_phi, g_cells, o_phi, o_cells, p.L) <= PHI_TOL_1
    # stored tile outside each active window stays exactly zero
    for n in range(6):
        wx, wy, tx0, ty0 = pfb200.CLASSES[int(g_cells["cls"][n])]
        t = g_phi[n].copy()
        t[ty0:ty0 + wy, tx0:tx0 + wx] = 0
        assert not t.any(), n
    # Q5.27 aggregate is exact given the stored field
    np.testing.assert_array_equal(g_S[:, :p.L], s_from_phi(g_phi, g_cells, p.L)[:, :p.L])
    np.testing.assert_array_equal(g_flags, o.flags())


def test_kernel_variants_agree(synth):
    p, cells, phi = synth
    out = {}
    for kv in KERNELS:
        ds = DeviceState2D(p, cells, phi, step=123)
        for _ in range(3):
            ds.step_with(launch_pfb(*kv))
        out[kv] = (ds.get_cells(), ds.get_phi(), ds.get_S())
    base = out[(4, 1)]
    for kv in KERNELS:
        assert_cells_match(out[kv][0], base[0], vel_rtol=1e-6, moment_rtol=1e-9)
        assert max_world_diff(out[kv][1], out[kv][0], base[1], base[0], p.L) <= 1e-6
        np.testing.assert_array_equal(out[kv][2][:, :p.L],
                                      s_from_phi(out[kv][1], out[kv][0], p.L)[:, :p.L])


@pytest.mark.parametrize("cluster,variant", [(2, 1), (4, 1), (8, 1)])
def test_deterministic_rerun(synth, cluster, variant):
    p, cells, phi = synth
    res = []
    for _ in range(2):
        ds = DeviceState2D(p, cells, phi, step=5)
        for _ in range(4):
            ds.step_with(launch_pfb(cluster, variant))
        res.append((ds.get_cells().tobytes(), ds.get_phi().tobytes(), ds.get_S().tobytes()))
    assert res[0] == res[1]


@pytest.mark.skipif(not oracle2d.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("cluster,variant", [(2, 1), (4, 1), (8, 1)])
def test_one_step_all_classes_vs_reference_kernel(synth, cluster, variant):
    p, cells, phi = synth
    step = 9000037
    a = DeviceState2D(p, cells, phi, step=step)
    a.step_with(launch_pfb(cluster, variant))
    b = DeviceState2D(p, cells, phi, step=step)
    b.step_with(launch_ref)
    ca, cb = a.get_cells(), b.get_cells()
    assert_cells_match(ca, cb, moment_rtol=1e-9)
    pa, pb = a.get_phi(), b.get_phi()
    d = max_world_diff(pa, ca, pb, cb, p.L)
    assert d <= PHI_TOL_1
    np.testing.assert_array_equal(a.get_flags(), b.get_flags())
    np.testing.assert_array_equal(a.get_S()[:, :p.L], s_from_phi(pa, ca, p.L)[:, :p.L])
    print(f"reference kernel vs pfb200, one step: max|dphi|={d:.3e}, "
          f"identical phi bits: {np.array_equal(pa, pb)}")


def c1_like_state(L=512, N=64, seed=1234):
    p = params(L, N, R=12.0, seed=seed)
    cx, cy = pfb200.palmieri_centres(N, L, 24.0, seed)
    cells, phi = oracle2d.init_state(p.to_c(), cx, cy, fresh_cells(p))
    return p, cells, phi


@pytest.mark.slow
def test_1000_steps_vs_oracle_and_fp64():
    p, cells, phi = c1_like_state()
    ds = DeviceState2D(p, cells, phi, step=0)
    for _ in range(1000):
        ds.step_with(launch_pfb(4, 1))
    g_cells, g_phi = ds.get_cells(), ds.get_phi()
    o32 = oracle_step(p, cells, phi, 0, n=1000)
    o_cells, o_phi = o32.cells(), o32.phi()
    d32 = max_world_diff(g_phi, g_cells, o_phi, o_cells, p.L)
    np.testing.assert_array_equal(g_cells["tumble_ctr"], o_cells["tumble_ctr"])
    np.testing.assert_array_equal(g_cells["theta"], o_cells["theta"])
    assert d32 <= PHI_TOL_1000, d32
    np.testing.assert_allclose(g_cells["V"], o_cells["V"], rtol=1e-6)
    o64 = oracle_step(p, cells, phi, 0, n=1000, f64=True)
    c64 = o64.cells()
    d64 = max_world_diff(g_phi, g_cells, o64.phi(), c64, p.L)
    v64 = o64.velocity()
    ev = np.abs(np.stack([g_cells["vx"], g_cells["vy"]], 1) - v64).max()
    eV = np.abs(g_cells["V"] - c64["V"]).max() / np.abs(c64["V"]).max()
    print(f"1000 steps: vs f32 oracle max|dphi|={d32:.3e}; vs f64 oracle max|dphi|={d64:.3e}, "
          f"max|dv|={ev:.3e}, max rel dV={eV:.3e}")
    assert d64 < 1e-3 and eV < 1e-4
    assert not pfb200.fatal(ds.get_flags())


@pytest.mark.slow
@pytest.mark.skipif(not oracle2d.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("cluster,variant", [(4, 1), (2, 1)])
def test_1000_steps_vs_reference_kernel(cluster, variant):
    p, cells, phi = c1_like_state()
    a = DeviceState2D(p, cells, phi, step=0)
    b = DeviceState2D(p, cells, phi, step=0)
    worst = {}
    for n in range(1, 1001):
        a.step_with(launch_pfb(cluster, variant))
        b.step_with(launch_ref)
        if n in (1, 10, 1000):
            ca, cb = a.get_cells(), b.get_cells()
            worst[n] = max_world_diff(a.get_phi(), ca, b.get_phi(), cb, p.L)
            np.testing.assert_array_equal(ca["tumble_ctr"], cb["tumble_ctr"])
            np.testing.assert_array_equal(ca["gx0"], cb["gx0"])
            np.testing.assert_allclose(ca["V"], cb["V"], rtol=1e-7)
            np.testing.assert_allclose(ca["vx"], cb["vx"], rtol=1e-4, atol=1e-8)
    print("reference kernel vs pfb200 max|dphi| after 1/10/1000 steps:", worst)
    assert worst[1] <= PHI_TOL_1 and worst[1000] <= PHI_TOL_1000


def test_sim_driver_graph_matches_launches():
    p, cells, phi = c1_like_state(L=320, N=12)
    s1 = pfb200.Sim2D(p, cells=cells, phi=phi, step=0, use_graph=True)
    s2 = pfb200.Sim2D(p, cells=cells, phi=phi, step=0, use_graph=False)
    s1.advance(13)
    s2.advance(13)
    assert s1.step == s2.step == 13
    assert s1.cells().tobytes() == s2.cells().tobytes()
    assert s1.phi().tobytes() == s2.phi().tobytes()
    assert s1.S().tobytes() == s2.S().tobytes()
    s1.close()
    s2.close()


def test_restart_equivalence():
    """3 steps equal 1+1+1 steps through state save/restore (the reference's
    restart contract, tests/run_gpu_smoke.py:67-109)."""
    p, cells, phi = c1_like_state(L=320, N=12)
    a = pfb200.Sim2D(p, cells=cells, phi=phi, step=0)
    a.advance(3)
    b = pfb200.Sim2D(p, cells=cells, phi=phi, step=0)
    for _ in range(3):
        b.advance(1)
        cb, pb, st = b.cells(), b.phi(), b.step
        b.close()
        b = pfb200.Sim2D(p, cells=cb, phi=pb, step=st)
    assert a.cells().tobytes() == b.cells().tobytes()
    assert a.phi().tobytes() == b.phi().tobytes()


def test_init_kernels_match_oracle():
    p = params(512, 64, R=12.0)
    cx, cy = pfb200.palmieri_centres(64, 512, 24.0, 99)
    s = pfb200.Sim2D(p, cx, cy)
    g_cells, g_phi = s.cells(), s.phi()
    o_cells, o_phi = oracle2d.init_state(p.to_c(), cx, cy, fresh_cells(p))
    np.testing.assert_array_equal(g_cells["gx0"], o_cells["gx0"])
    np.testing.assert_array_equal(g_cells["gy0"], o_cells["gy0"])
    np.testing.assert_array_equal(g_cells["theta"], o_cells["theta"])
    assert np.abs(g_phi - o_phi).max() <= 4e-7  # tanhf: device vs host libm, a few ulp
    np.testing.assert_allclose(g_cells["V"], o_cells["V"], rtol=1e-6)
    np.testing.assert_array_equal(s.S()[:, :512], s_from_phi(g_phi, g_cells, 512)[:, :512])
