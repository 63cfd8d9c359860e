"""Morton visit order of the 2D cells (the reference's --morton): the order
is the Z-order of each cell's centroid pixel, re-sorted every sixth step, and
it changes no result. The command line runs with --morton --no-l2 as the
reference's does."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pfb200

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell"
REF = ROOT / "oracle" / "_ref" / "cell_gh200"


def make_sim(use_graph=True):
    p = pfb200.SimParams2D(num_cells=37, L=512, target_radius=12.0, seed=3, v_A=0.05, tau=2.0)
    cx, cy = pfb200.palmieri_centres(37, 512, 24.0, 3)
    return pfb200.Sim2D(p, cx, cy, use_graph=use_graph)


def spread(v):
    v = v.astype(np.uint64) & np.uint64(0xFFFF)
    for s, m in ((8, 0x00FF00FF), (4, 0x0F0F0F0F), (2, 0x33333333), (1, 0x55555555)):
        v = (v | (v << np.uint64(s))) & np.uint64(m)
    return v


def morton_order(cells, L):
    """Cells by (Z-order of the truncated centroid pixel, index)."""
    V = np.where(cells["V"] > 0, cells["V"], 1.0)
    cx = np.mod(cells["gx0"] + np.trunc(cells["Cx"] / V).astype(np.int64), L)
    cy = np.mod(cells["gy0"] + np.trunc(cells["Cy"] / V).astype(np.int64), L)
    key = (spread(cx) | (spread(cy) << np.uint64(1))) << np.uint64(32)
    key |= np.arange(len(cells), dtype=np.uint64)
    return np.argsort(key, kind="stable").astype(np.uint32)


@pytest.mark.parametrize("use_graph", [True, False])
def test_morton_order_changes_nothing(use_graph):
    a, b = make_sim(use_graph), make_sim(use_graph)
    b.set_visit_order(True)
    for steps in (7, 12, 5):  # crosses the six-step sorting cadence off its grid
        a.advance(steps)
        b.advance(steps)
        a.sync()
        b.sync()
        np.testing.assert_array_equal(a.phi(), b.phi())
        assert a.cells().tobytes() == b.cells().tobytes()
        np.testing.assert_array_equal(a.flags(), b.flags())
    order = b.visit_order()
    assert not np.array_equal(order, np.arange(37, dtype=np.uint32))
    assert np.array_equal(np.sort(order), np.arange(37, dtype=np.uint32))
    b.set_visit_order(False)
    np.testing.assert_array_equal(b.visit_order(), np.arange(37, dtype=np.uint32))


def test_morton_order_is_the_centroid_z_order():
    sim = make_sim()
    sim.set_visit_order(True)
    np.testing.assert_array_equal(sim.visit_order(), morton_order(sim.cells(), 512))
    sim.advance(6)
    sim.sync()
    cells = sim.cells()  # the state the next step sorts
    sim.advance(1)
    sim.sync()
    np.testing.assert_array_equal(sim.visit_order(), morton_order(cells, 512))
    np.testing.assert_array_equal(sim.visit_order(), morton_order(cells, 512))


def rows(path):
    return Path(path).read_text().splitlines()


@pytest.mark.parametrize("exe", [EXE, REF])
def test_command_line_morton_same_trajectory(tmp_path, exe):
    if not exe.exists():
        pytest.skip("program not built")
    args = ("--N", 10, "--radius", 12, "--rho", 0.03, "--seed", 4, "--t-end", 0.3,
            "--trajectory-interval", 5, "--print-interval", 0, "--no-final-checkpoint")
    plain, morton = tmp_path / "plain.txt", tmp_path / "morton.txt"
    for out, extra in ((plain, ()), (morton, ("--morton", "--no-l2"))):
        r = subprocess.run([str(exe), *map(str, args), "--out", str(out), *extra], capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert rows(plain) == rows(morton)
    if exe == EXE and REF.exists():
        theirs = tmp_path / "theirs.txt"
        r = subprocess.run([str(REF), *map(str, args), "--out", str(theirs), "--morton"],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        a = np.array([[float(v) for v in ln.split()] for ln in rows(morton)[3:]])
        b = np.array([[float(v) for v in ln.split()] for ln in rows(theirs)[3:]])
        assert rows(morton)[:3] == rows(theirs)[:3]
        np.testing.assert_array_equal(a[:, :2], b[:, :2])
        np.testing.assert_allclose(a[:, 2:], b[:, 2:], rtol=0, atol=2e-6)
