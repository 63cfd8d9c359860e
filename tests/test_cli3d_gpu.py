"""pfb_cell_3d against the reference's own cell_gh200_3d (oracle/_ref) on the
same command line: identical trajectory metadata (centre-table hash,
realised density, measurement grouping), trajectory rows to the FP64
reduction-order tolerance, identical checkpoint parameter records and
bricks to 1e-5; each program resumes the other's checkpoint and appends to
the other's trajectory."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from pfb200 import checkpoint as ck

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell_3d"
REF = ROOT / "oracle" / "_ref" / "cell_gh200_3d"
ARGS = ("--N", 3, "--radius", 4, "--lambda", 3, "--v-A", 0.05, "--seed", 11,
        "--trajectory-interval", 2, "--print-interval", 0)
GEOMETRIES = [("periodic", 0.007), ("slab", 0.05), ("channel", 0.05)]


def run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r


def rows(path):
    lines = Path(path).read_text().splitlines()
    return lines[:2], np.array([[float(v) for v in ln.split()] for ln in lines[2:]])


def same_rows(a, b):
    """time and id exact; the rest within the FP64 moment reduction's
    grouping (positions, surface, volume) and binary32 rounding of the
    velocities that follow from them."""
    assert a.shape == b.shape
    np.testing.assert_array_equal(a[:, :2], b[:, :2])
    np.testing.assert_allclose(a[:, 2:5], b[:, 2:5], rtol=0, atol=1e-9)
    np.testing.assert_allclose(a[:, 5:], b[:, 5:], rtol=1e-6, atol=1e-9)


def same_checkpoint(pa, pb):
    a, b = ck.read3d(pa), ck.read3d(pb)
    assert a.step == b.step and a.brick_edge == b.brick_edge
    assert bytes(a.params) == bytes(b.params)
    assert a.base_measure_shards == b.base_measure_shards
    np.testing.assert_array_equal(a.cells["global_id"], b.cells["global_id"])
    np.testing.assert_allclose(a.phi, b.phi, rtol=0, atol=1e-5)
    return a


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
@pytest.mark.parametrize("geometry,rho", GEOMETRIES)
def test_same_command_line_same_outputs(tmp_path, geometry, rho):
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    args = (*ARGS, "--geometry", geometry, "--rho", rho, "--t-end", 0.04)
    run(EXE, *args, "--out", ours / "traj.txt", "--checkpoint-dir", ours)
    run(REF, *args, "--out", theirs / "traj.txt", "--checkpoint-dir", theirs)
    ha, ra = rows(ours / "traj.txt")
    hb, rb = rows(theirs / "traj.txt")
    assert ha == hb
    assert ra.shape[0] == 3 * 3  # frames at steps 0, 2, 4
    same_rows(ra, rb)
    assert same_checkpoint(ours / "checkpoint.pf3d", theirs / "checkpoint.pf3d").step == 4
    # each continues the other's run, appending to the other's trajectory
    run(EXE, "-c", theirs / "checkpoint.pf3d", "--t-end", 0.08, "--out", theirs / "traj.txt",
        "--checkpoint-dir", theirs / "next")
    run(REF, "-c", ours / "checkpoint.pf3d", "--t-end", 0.08, "--out", ours / "traj.txt",
        "--checkpoint-dir", ours / "next")
    ha, ra = rows(ours / "traj.txt")
    hb, rb = rows(theirs / "traj.txt")
    assert ha == hb and ra.shape[0] == 3 * 5
    same_rows(ra, rb)
    same_checkpoint(ours / "next" / "checkpoint.pf3d", theirs / "next" / "checkpoint.pf3d")


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
def test_tagged_and_rolling_checkpoints(tmp_path):
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    args = (*ARGS, "--rho", 0.007, "--t-end", 0.05, "--save-interval", 2, "--no-final-checkpoint")
    run(EXE, *args, "--checkpoint-dir", ours)
    run(REF, *args, "--checkpoint-dir", theirs)
    names = sorted(p.name for p in ours.iterdir())
    assert names == sorted(p.name for p in theirs.iterdir())
    assert names == ["checkpoint_000000000002.pf3d", "checkpoint_000000000004.pf3d"]
    for n in names:
        same_checkpoint(ours / n, theirs / n)


def test_append_refuses_another_run(tmp_path):
    run(EXE, *ARGS, "--rho", 0.007, "--t-end", 0.02, "--out", tmp_path / "traj.txt")
    args = (*ARGS[:-4], "--seed", 12, "--rho", 0.007, "--t-end", 0.02, "--out", tmp_path / "traj.txt")
    r = subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode != 0 and "does not match" in r.stderr


def test_resume_continues_the_sampling_grid(tmp_path):
    """A resumed leg keeps the file's absolute grid: frames at 0, 2, 4 from
    the first leg (t_end 0.05 ends at step 5, written as a closing frame),
    then 6 and 8."""
    d = tmp_path / "run"
    run(EXE, *ARGS, "--rho", 0.007, "--t-end", 0.05, "--out", d / "traj.txt", "--checkpoint-dir", d)
    _, r1 = rows(d / "traj.txt")
    np.testing.assert_allclose(np.unique(r1[:, 0]), [0.0, 0.02, 0.04, 0.05])
    run(EXE, "-c", d / "checkpoint.pf3d", "--t-end", 0.08, "--out", d / "traj.txt")
    _, r2 = rows(d / "traj.txt")
    np.testing.assert_allclose(np.unique(r2[:, 0]), [0.0, 0.02, 0.04, 0.05, 0.06, 0.08])


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
def test_initial_centres_table_same_run(tmp_path):
    """A periodic x,y,z centre table (side 49 for N=3, R=4, rho=0.007): both
    programs start from it and write the same header (its hash) and rows."""
    table = tmp_path / "c.csv"
    table.write_text("global_id,x,y,z\n0,24.5,24.5,24.5\n1,5.5,6.25,7\n2,40,40.5,10\n")
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    args = (*ARGS, "--rho", 0.007, "--t-end", 0.04, "--initial-centres", table)
    run(EXE, *args, "--out", ours / "traj.txt")
    run(REF, *args, "--out", theirs / "traj.txt")
    ha, ra = rows(ours / "traj.txt")
    hb, rb = rows(theirs / "traj.txt")
    assert ha == hb
    same_rows(ra, rb)


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
def test_soft_cells_same_run(tmp_path):
    """One soft cell of three (gamma 0.5): the same header (gamma_soft,
    soft_fraction), the same per-cell gamma column and rows, and identical
    checkpoint records; each continues the other's run."""
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    args = (*ARGS, "--rho", 0.007, "--t-end", 0.04, "--cancer-fraction", 0.34, "--gamma-cancer", 0.5)
    run(EXE, *args, "--out", ours / "traj.txt", "--checkpoint-dir", ours)
    run(REF, *args, "--out", theirs / "traj.txt", "--checkpoint-dir", theirs)
    ha, ra = rows(ours / "traj.txt")
    hb, rb = rows(theirs / "traj.txt")
    assert ha == hb and "soft_fraction=" in ha[0]
    np.testing.assert_array_equal(ra[:, 11], rb[:, 11])  # gamma per cell
    assert sorted(set(ra[:, 11])) == [0.5, 1.0]
    same_rows(ra, rb)
    same_checkpoint(ours / "checkpoint.pf3d", theirs / "checkpoint.pf3d")
    run(EXE, "-c", theirs / "checkpoint.pf3d", "--t-end", 0.06, "--out", theirs / "traj.txt")
    run(REF, "-c", ours / "checkpoint.pf3d", "--t-end", 0.06, "--out", ours / "traj.txt")
    ha, ra = rows(ours / "traj.txt")
    hb, rb = rows(theirs / "traj.txt")
    assert ha == hb
    same_rows(ra, rb)


@pytest.mark.parametrize("geometry,rho", GEOMETRIES)
def test_strict_verification_passes(tmp_path, geometry, rho):
    """--strict re-measures every 2 steps and requires the recorded volumes to
    hold to 1e-12 and no support on a brick face; a healthy run exits 0, as
    the reference's does."""
    args = (*ARGS, "--geometry", geometry, "--rho", rho, "--t-end", 0.06, "--strict",
            "--verify-every", 2)
    run(EXE, *args)
    if REF.exists():
        run(REF, *args)
