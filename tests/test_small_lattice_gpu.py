"""Lattice sides below the reference's minimum (it refuses L <= 286, its
largest window): here a side L >= 144 uses only the shape classes whose
window fits L, so no window overlaps itself on the periodic lattice. There
is no reference run to compare with, so the CPU oracle, which applies the
same class cap, is the check, in binary32 (phi within 1e-5 after 300 steps,
integer fields exact) and binary64 (errors per observable printed and
bounded). The 64-replica ensemble workload draws L = 256 among its sides.
"""
import numpy as np
import pytest

import oracle2d
import pfb200
from helpers2d import max_world_diff, params, synthetic_all_classes

pytestmark = pytest.mark.gpu


def dense_state(L, N, seed):
    p = params(L, N, R=12.0, seed=seed)
    cx, cy = oracle2d.palmieri_centres(N, L, 12.0, seed)
    cells, phi = oracle2d.init_state(p.to_c(), cx, cy, oracle2d.fresh_cells(p.to_c()))
    return p, cells, phi


@pytest.mark.parametrize("L,N", [(256, 96), (200, 40)])
def test_small_lattice_tracks_the_oracle(L, N):
    p, cells, phi = dense_state(L, N, 4242)
    sim = pfb200.Sim2D(p, cells=cells, phi=phi, step=0)
    sim.advance(300)
    g_cells, g_phi, g_flags = sim.cells(), sim.phi(), sim.flags()
    sim.close()
    o = oracle2d.OracleSim(p.to_c(), cells, phi, step=0)
    o.advance(300)
    oc, op, of = o.cells(), o.phi(), o.flags()
    o.close()
    for k in ("gx0", "gy0", "cls", "bb_lo_x", "bb_hi_x", "bb_lo_y", "bb_hi_y", "shift_ctr",
              "tumble_ctr"):
        np.testing.assert_array_equal(g_cells[k], oc[k], err_msg=k)
    np.testing.assert_array_equal(g_flags, of)
    assert not pfb200.fatal(g_flags)
    d32 = max_world_diff(g_phi, g_cells, op, oc, L)
    assert d32 <= 1e-5, d32
    o64 = oracle2d.OracleSim(p.to_c(), cells, phi, step=0, f64=True)
    o64.advance(300)
    c64 = o64.cells()
    d64 = max_world_diff(g_phi, g_cells, o64.phi(), c64, L)
    eV = float(np.max(np.abs(g_cells["V"] - c64["V"]) / c64["V"]))
    ev = float(np.max(np.abs(np.stack([g_cells["vx"], g_cells["vy"]], 1) - o64.velocity())))
    o64.close()
    print(f"L={L}, {N} cells, 300 steps: vs f32 oracle max|dphi|={d32:.2e}; vs f64 "
          f"max|dphi|={d64:.2e}, max rel dV={eV:.2e}, max|dv|={ev:.2e}")
    assert d64 <= 1e-4 and eV <= 1e-5


def test_class_cap_on_a_small_lattice():
    """A cell whose support needs a larger window than any fitting the side
    raises class_exhausted (the largest fitting window on 256 is class 4,
    224^2: the 286^2 fallback is not available), as in the oracle."""
    cells, phi = synthetic_all_classes(L=256)
    keep = [0, 1, 2, 3, 4]   # drop the class-5 cell: its window cannot fit
    cells, phi = cells[keep].copy(), phi[keep].copy()
    cells["global_id"] = np.arange(len(keep)) * 3 + 1
    cells[4]["bb_lo_x"], cells[4]["bb_hi_x"] = 1, 221  # extent 221 + 8 > 224
    p = params(256, len(keep), R=12.0, tau=0.02, full_moment_every=1)
    sim = pfb200.Sim2D(p, cells=cells, phi=phi, step=5)
    sim.advance(1)
    g_cells, g_flags = sim.cells(), sim.flags()
    sim.close()
    o = oracle2d.OracleSim(p.to_c(), cells, phi, step=5)
    o.advance(1)
    np.testing.assert_array_equal(g_flags, o.flags())
    assert g_flags[pfb200.FLAG_NAMES.index("class_exhausted")] >= 1
    np.testing.assert_array_equal(g_cells["cls"], o.cells()["cls"])
    o.close()
