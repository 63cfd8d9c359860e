"""The driver's default scatter (variants 0/1): the identity path adds q(phi)
into the Q5.27 aggregate with non-returning red.add, and S_overflow stays
exact through per-bin bounds recounted by the launch's last CTA. Checked on a
B200 against the returning scatter (variant 2) and against the reference's own
kernel (oracle/_ref/libref2d.so), which tests the value returned by every add
(src/kernels.cu:496-497):

* ordinary runs (lattice sides a multiple of 16 and not, full-moment steps,
  recentring shifts, a class change): phi, cells, aggregate and flags
  bit-identical between the two scatters;
* a host-built state whose aggregate really wraps (eight cells stacked on
  the same pixels): S_overflow raised, as by the reference kernel on the same state;
* a host-built state where one bin's bound passes 2^32 but no pixel's total
  does (ten cells with a bright pixel each, all in one bin): the exact recount
  runs and raises nothing, as the reference raises nothing.
"""
import ctypes as C

import numpy as np
import pytest

import oracle2d
import pfb200
from pfb200 import CELL_DTYPE
from helpers2d import DeviceState2D, params, s_from_phi, synthetic_all_classes

pytestmark = pytest.mark.gpu

S_OVERFLOW = pfb200.FLAG_NAMES.index("S_overflow")


def run_sim(p, cells, phi, steps, variant, step=0):
    s = pfb200.Sim2D(p, cells=cells, phi=phi, step=step, use_graph=True, variant=variant)
    s.advance(steps)
    out = (s.cells(), s.phi(), s.S(), s.flags(), s.scatter_recounts())
    s.close()
    return out


def c1_state(L, N, seed):
    p = params(L, N, R=12.0, seed=seed)
    cx, cy = pfb200.palmieri_centres(N, L, 24.0, seed)
    cells, phi = oracle2d.init_state(p.to_c(), cx, cy, oracle2d.fresh_cells(p.to_c()))
    return p, cells, phi


@pytest.mark.parametrize("L,N,steps", [(512, 64, 210), (701, 40, 130), (2048, 1024, 12)])
def test_binned_scatter_equals_returning_scatter(L, N, steps):
    p, cells, phi = c1_state(L, N, 17)
    a = run_sim(p, cells, phi, steps, 0)
    b = run_sim(p, cells, phi, steps, 2)
    assert a[0].tobytes() == b[0].tobytes()
    assert a[1].tobytes() == b[1].tobytes()
    assert a[2].tobytes() == b[2].tobytes()
    np.testing.assert_array_equal(a[3], b[3])
    assert a[4] == 0  # ordinary states never reach a bound of 2^32
    assert int(a[0]["shift_ctr"].sum()) > 0


def test_binned_scatter_all_classes():
    cells, phi = synthetic_all_classes(L=701)
    p = params(701, 6, R=12.0, tau=0.02, full_moment_every=7)
    a = run_sim(p, cells, phi, 9, 0, step=123)
    b = run_sim(p, cells, phi, 9, 2, step=123)
    for x, y in zip(a[:3], b[:3]):
        assert x.tobytes() == y.tobytes()
    np.testing.assert_array_equal(a[3], b[3])


def stacked_state(spread: bool, L=704):
    """Class-0 cells. spread=False: eight cells each hold a 3x3 block of
    phi = 1.99 on the same lattice pixels; their aggregate stays below 2^32
    (8 q(1.99) = 4.25e9), but the step drives every |phi| there past 2, and
    8 * 2^29 = 2^32 wraps. spread=True: ten cells each hold one pixel of
    phi = 2 at its own lattice pixel, all inside one 16 x 16 bin: the bin's
    bound passes 2^32 (10 x ~4.8e8) while every total stays near 4.8e8."""
    n = 10 if spread else 8
    cells = np.zeros(n, CELL_DTYPE)
    phi = np.zeros((n, 288, 288), np.float32)
    for k in range(n):
        c = cells[k]
        c["global_id"] = k
        c["gamma"], c["v_A"], c["R_tgt"], c["M_pf"], c["theta"] = 1.0, 0.01, 12.0, 0.5, 0.1 * k
        # window pixel (72, 72) sits at lattice (321 + k, 323 + k) or (330, 330)
        X, Y = (321 + k, 323 + k) if spread else (330, 330)
        c["gx0"], c["gy0"] = X - 72, Y - 72
        if spread:
            phi[k, 64 + 72, 64 + 72] = 2.0
        else:
            phi[k, 64 + 71:64 + 74, 64 + 71:64 + 74] = 1.99
        w = phi[k, 64:208, 64:208].astype(np.float64)
        d = w * w
        yy, xx = np.mgrid[0:144, 0:144]
        c["V"], c["Cx"], c["Cy"] = d.sum(), (d * xx).sum(), (d * yy).sum()
        sup = np.argwhere(w > 1e-5)
        c["bb_lo_y"], c["bb_lo_x"] = sup.min(0)
        c["bb_hi_y"], c["bb_hi_x"] = sup.max(0)
        c["phi_max"] = np.abs(w).max()
    return params(L, n, R=12.0, seed=5), cells, phi


def reference_step(p, cells, phi):
    ds = DeviceState2D(p, cells, phi, step=0)
    ds.step_with(lambda a: oracle2d.rlib().ref2d_launch_step(C.byref(a),
                                                             oracle2d.rlib().ref2d_grid(0), None))
    return ds.get_cells(), ds.get_phi(), ds.get_flags()


@pytest.mark.parametrize("spread", [False, True], ids=["wraps", "bound-only"])
def test_overflow_detection_matches_returning_scatter_and_reference(spread):
    p, cells, phi = stacked_state(spread)
    a = run_sim(p, cells, phi, 1, 0)
    b = run_sim(p, cells, phi, 1, 2)
    assert a[1].tobytes() == b[1].tobytes()
    np.testing.assert_array_equal(a[3], b[3])
    assert a[4] >= 1, "the bin's bound should have reached 2^32 and been recounted"
    assert bool(a[3][S_OVERFLOW]) == (not spread)
    if not spread:
        # the stored field's exact totals do wrap somewhere
        S64 = np.zeros((p.L, p.L), np.int64)
        for n in range(len(a[0])):
            t = a[1][n, 64:208, 64:208].astype(np.float32)
            q = np.rint(np.minimum(t * t, np.float32(4)) * np.float32(2**27)).astype(np.int64)
            gy = (a[0]["gy0"][n] + np.arange(144)) % p.L
            gx = (a[0]["gx0"][n] + np.arange(144)) % p.L
            S64[np.ix_(gy, gx)] += q
        assert S64.max() >= 2**32
    if oracle2d.ref_available():
        rc, rp, rf = reference_step(p, cells, phi)
        assert rp.tobytes() == a[1].tobytes()
        np.testing.assert_array_equal(rf, a[3])
