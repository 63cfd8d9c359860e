"""Pin the oracle (and the library's host primitives) to the reference's own
known answers:

* Philox4x32-10 vectors of tests/common_primitives_cpu_test.cpp:54-61;
* the bitwise coefficient identities of tests/common_primitives_cpu_test.cpp:24-52;
* the phase-field RHS cases of tests/mobility_model_cpu_test.cpp:44-151
  (default path == the pre-mobility expression bit for bit; the mobility
  scales exactly the passive part; advection is independent of it).

Arithmetic here uses numpy float32/float64 scalars, which round every
operation separately (no contraction), like the reference's host build.
"""
import numpy as np
import pytest

import oracle2d
import pfb200

F = np.float32

PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((1, 2, 3, 4), (5, 6), (0xC0C839BC, 0x889C87C5, 0x61986739, 0x2D4623D0)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
]


@pytest.mark.parametrize("ctr,key,expect", PHILOX_KAT)
def test_philox_known_answers_oracle(ctr, key, expect):
    assert tuple(oracle2d.philox(ctr, key)) == expect


@pytest.mark.parametrize("ctr,key,expect", PHILOX_KAT)
def test_philox_known_answers_library_host(ctr, key, expect):
    import ctypes as C
    out = (C.c_uint32 * 4)()
    pfb200.lib().pfb_philox4x32_10(*ctr, *key, out)
    assert tuple(out) == expect


def test_uniform53():
    L = oracle2d.olib()
    assert L.oracle_u53(0, 0) == 0.0
    assert L.oracle_u53(0xFFFFFFFF, 0xFFFFFFFF) == (2**53 - 1) / 2**53
    assert L.oracle_u53(0x80000000, 0) == 0.5
    assert pfb200.lib().pfb_philox_uniform53(0x12345678, 0x9ABCDEF0) == \
        L.oracle_u53(0x12345678, 0x9ABCDEF0)


COEFF_SETS = [  # (lambda, kappa, xi, mu, target, f64)
    (7.0, 10.0, 1500.0, 1.0, 7542.0, False),
    (5.25, 3.7, 977.0, 0.125, 11.75, False),
    (7.0, 10.0, 1500.0, 1.0, 7542.0, True),
    (0.5, 0.125, 65536.0, 3.7, 0.75, True),
]


@pytest.mark.parametrize("lam,kappa,xi,mu,target,f64", COEFF_SETS)
def test_coefficient_bit_identities(lam, kappa, xi, mu, target, f64):
    T = np.float64 if f64 else np.float32
    lam, kappa, xi, mu, target = (T(v) for v in (lam, kappa, xi, mu, target))
    got = oracle2d.coefficients(lam, kappa, xi, mu, target, f64)
    k = T(2.7386127875258306) / lam
    want = [T(30) / (lam * lam), T(60) * kappa / (lam * lam),
            (T(60) * kappa / (lam * lam)) / xi, T(2) * mu / target, k, target + T(0.5) / k]
    for g, w in zip(got, want):
        assert T(g).tobytes() == T(w).tobytes()


PIXELS = [
    (0.125, 0.5, 0.25, 0.03, -0.02),
    (-0.75, 0.9999, 0.0, -0.4, 0.4),
    (2.5e-3, 1.0e-5, 0.9, 1.0e-4, -1.0e-4),
    (-3.1, 0.31, 1.7, 0.11, 0.07),
    (0.0, 0.0, 0.0, 0.0, 0.0),
    (1.0, 1.0, 1.0, 1.0, 1.0),
    (-1.9e-4, 0.62, 3.9, -0.9, -0.8),
]
COEFFS = [  # gam, dwC, volC, repC, vx, vy
    (1.0, 0.612244879, 1.3e-4, 12.2448978, 0.01, -0.02),
    (0.35, 0.214285716, -2.0e-4, 12.2448978, -0.004, 0.006),
    (2.0, 1.5, 0.5, 0.0, 0.0, 0.3),
]


def legacy_rhs(lap, phi, So, gx, gy, gam, dwC, volC, repC, vx, vy):
    one, two = F(1), F(2)
    return (gam * lap - dwC * (phi * (one - phi) * (one - two * phi)) + volC * phi
            - repC * phi * So - (vx * gx + vy * gy))


def rhs(*a):
    return F(oracle2d.olib().oracle_rhs_f32(*[float(F(v)) for v in a]))


def bits(x):
    return F(x).tobytes()


@pytest.mark.parametrize("px", PIXELS)
@pytest.mark.parametrize("co", COEFFS)
def test_rhs_default_path_bitwise(px, co):
    a = [F(v) for v in px + co]
    assert bits(rhs(*a, F(1))) == bits(legacy_rhs(*a))


@pytest.mark.parametrize("px", PIXELS)
@pytest.mark.parametrize("co", COEFFS)
@pytest.mark.parametrize("mrel", [0.5, 1.0 / 0.35, 2.857143, 4.0])
def test_rhs_mobility_scales_passive_only(px, co, mrel):
    lap, phi, So, gx, gy = (F(v) for v in px)
    gam, dwC, volC, repC, vx, vy = (F(v) for v in co)
    mrel = F(mrel)
    p1 = rhs(lap, phi, So, gx, gy, gam, dwC, volC, repC, F(0), F(0), F(1))
    pm = rhs(lap, phi, So, gx, gy, gam, dwC, volC, repC, F(0), F(0), mrel)
    assert bits(pm) == bits(mrel * p1)
    adv = vx * gx + vy * gy
    full = rhs(lap, phi, So, gx, gy, gam, dwC, volC, repC, vx, vy, mrel)
    assert bits(full) == bits(pm - adv)


@pytest.mark.parametrize("px", PIXELS)
def test_rhs_advection_independent_of_mobility(px):
    lap, phi, So, gx, gy = (F(v) for v in px)
    z = F(0)
    a1 = rhs(lap, phi, So, gx, gy, z, z, z, z, F(0.013), F(-0.021), F(1))
    a2 = rhs(lap, phi, So, gx, gy, z, z, z, z, F(0.013), F(-0.021), F(1 / 0.35))
    assert bits(a1) == bits(a2)


def test_q_of_encoding():
    L = oracle2d.olib()
    lib = pfb200.lib()
    for v in [0.0, 1e-5, 6.1e-5, 0.1, 0.5, 0.9999, 1.0, 1.5, 2.0, 3.0, -0.7, float("nan")]:
        sq = min(F(v) * F(v), F(4)) if v == v else F(4)
        want = int(np.rint(np.float64(F(sq * F(2**27)))))
        assert L.oracle_q_of(v) == want
        assert lib.pfb_q_of(v) == want


# ---- fresh-start draws: the oracle against the reference's own host code ----
@pytest.mark.skipif(not oracle2d.ref_available(), reason="reference build absent")
def test_oracle_ic_draws_equal_reference():
    r = oracle2d.rlib()
    o = oracle2d.olib()
    for gid in (0, 1, 7, 1023, 123456, 2**31 - 1):
        for stream in (1234, 0xDEADBEEFCAFEF00D, 1):
            assert o.oracle_ic_theta(gid, stream) == r.ref2d_ic_theta(gid, stream)
            for sigma in (0.0, 0.3, 1.2):
                assert o.oracle_ic_v_A(gid, stream, 0.01, sigma) == \
                    r.ref2d_ic_v_A(gid, stream, 0.01, sigma)


@pytest.mark.skipif(not __import__("oracle3d").ref_cpu_available(),
                    reason="reference host build absent")
@pytest.mark.parametrize("n,side,sep,seed", [(64, 512.0, 24.0, 1234), (1024, 2048.0, 24.0, 1234),
                                             (187, 256.0, 10.0, 99)])
def test_oracle_placement_equals_reference(n, side, sep, seed):
    import ctypes as C
    import oracle3d
    x, y = oracle2d.palmieri_centres(n, side, sep, seed)
    rx, ry = np.zeros(n, np.float32), np.zeros(n, np.float32)
    fp = C.POINTER(C.c_float)
    assert oracle3d.rclib().ref3d_cpu_palmieri2d(n, side, sep, seed, rx.ctypes.data_as(fp),
                                                 ry.ctypes.data_as(fp)) == 0
    np.testing.assert_array_equal(x, rx)
    np.testing.assert_array_equal(y, ry)


def test_oracle_fresh_cells_equal_library():
    from helpers2d import fresh_cells, params
    p = params(512, 64, R=12.0, seed=77, v_A_sigma=0.4, cancer_fraction=0.25)
    a = oracle2d.fresh_cells(p.to_c())
    b = fresh_cells(p)
    assert a.tobytes() == b.tobytes()
