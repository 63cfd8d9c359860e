"""16-bit phi pools in 3D (binary16 / bfloat16 storage, binary32 arithmetic,
stochastic rounding) on a B200: the binary32 pools stay bit-identical to
the plain driver; the 16-bit runs are reproducible, keep their integrity
flags clear and are compared with the FP64 oracle (oracle/pf3d_oracle.cpp)
per observable after 100 steps at the benchmarked lambda 7, R 10, B 64
(128^3, 64 cells). The errors are printed and bounded by the storage's
resolution. The Q5.27 aggregate of every 16-bit run equals the exact
integer restatement of its own stored field."""
import numpy as np
import pytest

import oracle3d
import pfb200
from test_bench_config_parity_gpu import c3_centres, c3_params, world_diff3d

pytestmark = pytest.mark.gpu


def q_total(p, sim):
    """Exact aggregate rebuilt from the stored field (binary32 values of the
    16-bit pool) with the Q5.27 rule, through the oracle's integer scatter."""
    import ctypes as C
    phi = np.ascontiguousarray(sim.phi(), np.float32)
    cells = np.ascontiguousarray(sim.cells())
    S = np.zeros_like(sim.S())
    flags = np.zeros(10, np.uint32)
    oracle3d.olib().oracle3d_scatter(0, oracle3d._p(phi), oracle3d._p(cells), oracle3d._p(S),
                                     oracle3d._p(flags), C.byref(sim.layout), len(cells), sim.B)
    return S


def run(p, c, steps, storage, **kw):
    p.phi_storage = storage
    s = pfb200.Sim3D(p, c, **kw)
    s.advance(steps)
    return s


@pytest.mark.parametrize("storage", [1, 2], ids=["binary16", "bfloat16"])
def test_16bit_pools_against_fp64_oracle(storage):
    p = c3_params("periodic", 64, 128, 128)
    p.full_moment_every = 0
    c = c3_centres(p)
    f32 = run(p, c, 0, 0)
    o64 = oracle3d.OracleState3D(p, f32.layout, f32.B, f32.cells(), f32.phi(), f32.S(), f64=True)
    f32.close()
    steps = 100
    a = run(p, c, steps, storage)
    b = run(p, c, steps, storage)
    assert o64.advance(steps) == [0] * steps
    ca, cb, co = a.cells(), b.cells(), o64.cells
    # reproducible: the rounding stream is a hash of (seed, step, cell, voxel)
    assert a.phi().tobytes() == b.phi().tobytes() and ca.tobytes() == cb.tobytes()
    assert not a.flags().any()
    # a cell near a half-voxel recentring threshold may shift one step apart
    # from the FP64 run: compare in world coordinates
    moved = sum(int(np.count_nonzero(ca["origin_" + k] != co["origin_" + k])) for k in "xyz")
    assert moved <= 4, moved
    e_phi = world_diff3d(a.phi().astype(np.float64), ca, o64.phi, co)
    e_V = float(np.max(np.abs(ca["V"] - co["V"]) / co["V"]))
    cen = lambda x, k: x["origin_" + k] + x["C" + k] / x["V"]  # noqa: E731
    e_C = max(float(np.max(np.abs(cen(ca, k) - cen(co, k)))) for k in "xyz")
    vel = lambda x: np.stack([x["velocity_" + k] for k in "xyz"], 1).astype(np.float64)  # noqa: E731
    e_v = float(np.max(np.abs(vel(ca) - vel(co)))) / p.v_A
    name = {1: "binary16", 2: "bfloat16"}[storage]
    print(f"C3 {name} pools (128^3, 64 cells, B=64) after {steps} steps vs the FP64 oracle: "
          f"max|dphi|={e_phi:.2e} max rel dV={e_V:.2e} max|dC|={e_C:.2e} max|dv|/v_A={e_v:.2e}")
    # the bounds of the 2D 16-bit pools: a few storage ulps of phi ~ 1
    # (binary16 9.8e-4, bfloat16 7.8e-3), moments and motion well below the
    # cells' own change
    lim = {1: dict(phi=2e-2, V=2e-3, C=5e-2, v=5e-2), 2: dict(phi=1e-1, V=2e-2, C=3e-1, v=3e-1)}[storage]
    assert e_phi <= lim["phi"] and e_V <= lim["V"] and e_C <= lim["C"] and e_v <= lim["v"]
    np.testing.assert_array_equal(a.S(), q_total(p, a))
    a.close()
    b.close()


@pytest.mark.parametrize("geometry", ["periodic", "slab", "channel"])
def test_16bit_pools_run_in_every_geometry_and_mode(geometry):
    from helpers3d import small_centres, small_params
    p = small_params(geometry)
    c = small_centres(p)
    ref = run(p, c, 25, 1)
    comp = run(p, c, 25, 1, memory_mode="compact", scratch_slots=4)
    assert ref.phi().tobytes() == comp.phi().tobytes()
    assert ref.cells().tobytes() == comp.cells().tobytes()
    np.testing.assert_array_equal(ref.S(), comp.S())
    assert not ref.flags().any()
    np.testing.assert_array_equal(ref.S(), q_total(p, ref))
    # the binary32 driver is unchanged by the pool type machinery
    f = run(p, c, 25, 0)
    g = run(p, c, 25, 0, memory_mode="balanced")
    assert f.phi().tobytes() == g.phi().tobytes()
    for s in (ref, comp, f, g):
        s.close()
