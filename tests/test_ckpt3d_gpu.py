"""3D checkpoints on the GPU: a restart through a PF3D file written here
continues exactly as the uninterrupted run, in all three geometries, and
files cross between this library and the reference's own cell_gh200_3d
(built from the reference sources in oracle/_ref) in both directions
(reference restore: src/pf3d/sim.cu:794-885)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pfb200
from helpers3d import small_centres, small_params
from pfb200 import checkpoint as ck

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "cell_gh200_3d"
EXACT = ("global_id", "origin_x", "origin_y", "origin_z", "bb_lo_x", "bb_hi_x", "bb_lo_y",
         "bb_hi_y", "bb_lo_z", "bb_hi_z", "pending_shift_x", "pending_shift_y", "pending_shift_z",
         "gamma", "v_A", "R_tgt")


@pytest.mark.parametrize("geometry", ["periodic", "slab", "channel"])
def test_restart_through_a_pf3d_file(tmp_path, geometry):
    p = small_params(geometry)
    a = pfb200.Sim3D(p, small_centres(p))
    c = pfb200.Sim3D(p, small_centres(p))  # never written
    a.advance(3)
    path = tmp_path / "c.pf3d"
    ck.write_sim3d(a, path)  # measures the current state first
    b = ck.restart3d(path)
    assert b.step == 3 and b.B == a.B
    a.advance(4)
    b.advance(4)
    c.advance(7)
    assert a.step == b.step == c.step == 7
    np.testing.assert_array_equal(a.phi(), b.phi())
    np.testing.assert_array_equal(a.phi(), c.phi())
    c.close()
    ca, cb = a.cells(), b.cells()
    for f in EXACT + ("V", "Cx", "Cy", "Cz", "Ix", "velocity_x", "polarity_x", "tumble_ctr"):
        np.testing.assert_array_equal(ca[f], cb[f], err_msg=f)
    assert a.S().tobytes() == b.S().tobytes()
    a.close()
    b.close()


def run_ref(*args):
    r = subprocess.run([str(REF), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def close_state(ours, theirs_cells, theirs_phi):
    """phi to 1e-5 (the measured FP64 moments, and so the binary32
    velocities, may differ from the reference's in the last bits: different
    reduction order), integer state exactly, FP64 moments to 1e-9. Both sides
    are measured on the current state (the reference measures before it
    writes)."""
    ours.measure_current()
    oc, op = ours.cells(), ours.phi()
    for f in EXACT:
        np.testing.assert_array_equal(oc[f], theirs_cells[f], err_msg=f)
    np.testing.assert_allclose(op, theirs_phi, rtol=0, atol=1e-5)
    for f in ("V", "Cx", "Cy", "Cz"):
        np.testing.assert_allclose(oc[f], theirs_cells[f], rtol=1e-9, err_msg=f)


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
def test_files_cross_between_reference_and_library(tmp_path):
    d1, d2, d3 = tmp_path / "d1", tmp_path / "d2", tmp_path / "d3"
    common = ("--radius", 4, "--lambda", 3, "--v-A", 0.05)
    run_ref("--N", 3, "--rho", 0.007, "--seed", 11, "--t-end", 0.04, "--checkpoint-dir", d1,
            "--print-interval", 0, *common)
    first = ck.read3d(d1 / "checkpoint.pf3d")
    assert first.cells.size == 3 and first.step > 0
    ours = ck.restart3d(d1 / "checkpoint.pf3d")
    run_ref("-c", d1 / "checkpoint.pf3d", "--t-end", 0.08, "--checkpoint-dir", d2,
            "--print-interval", 0)
    theirs = ck.read3d(d2 / "checkpoint.pf3d")
    ours.advance(theirs.step - ours.step)
    close_state(ours, theirs.cells, theirs.phi)
    mine = tmp_path / "mine.pf3d"
    ck.write_sim3d(ours, mine, first.params)
    run_ref("-c", mine, "--t-end", 0.12, "--checkpoint-dir", d3, "--print-interval", 0)
    theirs = ck.read3d(d3 / "checkpoint.pf3d")
    ours.advance(theirs.step - ours.step)
    close_state(ours, theirs.cells, theirs.phi)
    ours.close()
