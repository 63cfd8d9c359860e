"""2D checkpoints on the GPU: restart through a file written here is
equivalent to continuing in memory, and files cross between this library and
the reference's own cell_gh200 (built from the reference sources in
oracle/_ref) in both directions with bit-identical continuations (the step
kernels are bit-identical; reference restart contract: tests/run_gpu_smoke.py:
67-109, src/sim.cu:375-470)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pfb200
from helpers2d import params
from pfb200 import checkpoint as ck

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "cell_gh200"
EXACT = ("gx0", "gy0", "cls", "bb_lo_x", "bb_hi_x", "bb_lo_y", "bb_hi_y", "phi_max", "theta",
         "gamma", "v_A", "R_tgt", "M_pf", "promote_ctr")


def same_state(a_cells, a_phi, b_cells, b_phi):
    """phi and the integer / copied fields bit for bit; the FP64 moment sums
    to 1e-14 (their reduction order differs from the reference's by design),
    the binary32 velocity derived from them to 1e-6."""
    np.testing.assert_array_equal(a_phi, b_phi)
    for f in EXACT:
        np.testing.assert_array_equal(a_cells[f], b_cells[f], err_msg=f)
    for f in ("V", "Cx", "Cy"):
        np.testing.assert_allclose(a_cells[f], b_cells[f], rtol=1e-14, err_msg=f)
    for f in ("vx", "vy"):
        np.testing.assert_allclose(a_cells[f], b_cells[f], rtol=1e-6, atol=1e-12, err_msg=f)


def test_restart_through_a_checkpoint_file(tmp_path):
    p = params(320, 12, R=12.0, seed=8)
    cx, cy = pfb200.palmieri_centres(12, 320, 24.0, 8)
    a = pfb200.Sim2D(p, cx, cy)
    a.advance(5)
    path = tmp_path / "c.bin"
    ck.write_sim(a, path)
    b = ck.restart(path)
    assert b.step == 5
    a.advance(7)
    b.advance(7)
    same_state(a.cells(), a.phi(), b.cells(), b.phi())
    assert a.S().tobytes() == b.S().tobytes()
    a.close()
    b.close()


def run_ref(*args):
    r = subprocess.run([str(REF), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
def test_files_cross_between_reference_and_library(tmp_path):
    d1, d2, d3 = tmp_path / "d1", tmp_path / "d2", tmp_path / "d3"
    run_ref("--N", 8, "--radius", 12, "--rho", 0.03, "--seed", 5, "--t-end", 0.05,
            "--checkpoint-dir", d1)
    first = ck.read(d1 / "checkpoint.bin")
    assert first.cells.size == 8 and first.step > 0
    # the reference's file, continued here and by the reference
    ours = ck.restart(d1 / "checkpoint.bin")
    run_ref("-c", d1 / "checkpoint.bin", "--t-end", 0.1, "--checkpoint-dir", d2)
    theirs = ck.read(d2 / "checkpoint.bin")
    ours.advance(theirs.step - ours.step)
    same_state(ours.cells(), ours.phi(), theirs.cells, theirs.phi)
    # a file written here, continued by the reference and here
    mine = tmp_path / "mine.bin"
    ck.write_sim(ours, mine, first.params)
    run_ref("-c", mine, "--t-end", 0.15, "--checkpoint-dir", d3)
    theirs = ck.read(d3 / "checkpoint.bin")
    ours.advance(theirs.step - ours.step)
    same_state(ours.cells(), ours.phi(), theirs.cells, theirs.phi)
    assert not pfb200.fatal(ours.flags())
    ours.close()
