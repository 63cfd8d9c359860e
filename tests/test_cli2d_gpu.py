"""pfb_cell against the reference's own cell_gh200 (oracle/_ref) on the same
command line: identical trajectory header (metadata, centre-table hash),
trajectory rows, and final checkpoints with bit-identical phi; a run resumed
by one from the other's checkpoint appends to the other's trajectory."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from pfb200 import checkpoint as ck

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell"
REF = ROOT / "oracle" / "_ref" / "cell_gh200"
ARGS = ("--N", 8, "--radius", 12, "--rho", 0.03, "--seed", 5, "--trajectory-interval", 5,
        "--print-interval", 0)


def run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r


def rows(path):
    lines = Path(path).read_text().splitlines()
    head = lines[:3]
    data = np.array([[float(v) for v in ln.split()] for ln in lines[3:]])
    return head, data


def same_rows(a, b):
    assert a.shape == b.shape
    np.testing.assert_array_equal(a[:, :2], b[:, :2])        # time, cell id
    np.testing.assert_allclose(a[:, 2:], b[:, 2:], rtol=0, atol=2e-6)


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
def test_same_command_line_same_outputs(tmp_path):
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    run(EXE, *ARGS, "--t-end", 0.2, "--out", ours / "traj.txt", "--checkpoint-dir", ours)
    run(REF, *ARGS, "--t-end", 0.2, "--out", theirs / "traj.txt", "--checkpoint-dir", theirs)
    ha, ra = rows(ours / "traj.txt")
    hb, rb = rows(theirs / "traj.txt")
    assert ha == hb
    assert ra.shape[0] == 8 * 4
    same_rows(ra, rb)
    a, b = ck.read(ours / "checkpoint.bin"), ck.read(theirs / "checkpoint.bin")
    assert a.step == b.step == 20
    np.testing.assert_array_equal(a.phi, b.phi)
    assert bytes(a.params) == bytes(b.params)
    # each continues the other's run, appending to the other's trajectory
    run(EXE, "-c", theirs / "checkpoint.bin", "--t-end", 0.3, "--out", theirs / "traj.txt",
        "--checkpoint-dir", theirs / "next")
    run(REF, "-c", ours / "checkpoint.bin", "--t-end", 0.3, "--out", ours / "traj.txt",
        "--checkpoint-dir", ours / "next")
    ha, ra = rows(ours / "traj.txt")
    hb, rb = rows(theirs / "traj.txt")
    assert ha == hb and ra.shape[0] == 8 * 6
    same_rows(ra, rb)
    a, b = ck.read(ours / "next" / "checkpoint.bin"), ck.read(theirs / "next" / "checkpoint.bin")
    np.testing.assert_array_equal(a.phi, b.phi)


def test_append_refuses_another_run(tmp_path):
    run(EXE, *ARGS, "--t-end", 0.1, "--out", tmp_path / "traj.txt")
    args = ("--N", 8, "--radius", 12, "--rho", 0.03, "--seed", 6, "--t-end", 0.1,
            "--out", tmp_path / "traj.txt")
    r = subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode != 0 and "does not match" in r.stderr


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
def test_initial_centres_table_same_run(tmp_path):
    """A validated x,y centre table: both programs start from it and write the
    same trajectory header (its hash) and rows."""
    import pfb200
    L = pfb200.domain_side_for(8, 12, 0.03)
    c = L / 2
    pts = [(c, c), (20.5, 30.0), (100.0, 40.0), (150.25, 200.0), (30.0, 150.0), (260.0, 260.0),
           (200.0, 100.0), (80.0, 250.0)]
    table = tmp_path / "c.csv"
    table.write_text("global_id,x,y\n" + "".join(f"{i},{x!r},{y!r}\n" for i, (x, y) in enumerate(pts)))
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    run(EXE, *ARGS, "--t-end", 0.2, "--initial-centres", table, "--out", ours / "traj.txt")
    run(REF, *ARGS, "--t-end", 0.2, "--initial-centres", table, "--out", theirs / "traj.txt")
    ha, ra = rows(ours / "traj.txt")
    hb, rb = rows(theirs / "traj.txt")
    assert ha == hb
    same_rows(ra, rb)


def test_strict_reports_invariants(tmp_path):
    args = (*ARGS, "--t-end", 0.2, "--strict", "--verify-every", 5)
    r = subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if "[verify]" in ln]
    assert len(lines) == 4  # steps 5, 10, 15, 20
    for ln in lines:
        rel = float(ln.split("max rel V error")[1].split()[0])
        assert rel < 1e-12


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
def test_mobility_map_same_run(tmp_path):
    """Per-cell mobilities from a map: the same trajectory and bit-identical
    checkpoints (fields and stored mobilities) as cell_gh200; on resume the
    map overrides only its listed cells in both programs."""
    m = tmp_path / "m.txt"
    m.write_text("1 0.25\n3 1.0\n")
    m2 = tmp_path / "m2.txt"
    m2.write_text("5 0.125\n")
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    for exe, d in ((EXE, ours), (REF, theirs)):
        run(exe, *ARGS, "--t-end", 0.2, "--phase-field-mobility-map", m, "--out", d / "traj.txt",
            "--checkpoint-dir", d)
    ha, ra = rows(ours / "traj.txt")
    hb, rb = rows(theirs / "traj.txt")
    assert ha == hb
    same_rows(ra, rb)
    a, b = ck.read(ours / "checkpoint.bin"), ck.read(theirs / "checkpoint.bin")
    np.testing.assert_array_equal(a.phi, b.phi)
    np.testing.assert_array_equal(a.cells["M_pf"], b.cells["M_pf"])
    assert sorted(set(a.cells["M_pf"])) == [0.25, 0.5, 1.0]
    for exe, d in ((EXE, ours), (REF, theirs)):
        run(exe, "-c", d / "checkpoint.bin", "--t-end", 0.3, "--phase-field-mobility-map", m2,
            "--checkpoint-dir", d / "next")
    a, b = ck.read(ours / "next" / "checkpoint.bin"), ck.read(theirs / "next" / "checkpoint.bin")
    np.testing.assert_array_equal(a.phi, b.phi)
    np.testing.assert_array_equal(a.cells["M_pf"], b.cells["M_pf"])
    assert sorted(set(a.cells["M_pf"])) == [0.125, 0.25, 0.5, 1.0]
