"""PFB boundary recorder of the 2D system (reference src/boundary.cu).

Each frame is checked against a numpy restatement on the same state: the
cell records (tile origin, periodic centroid, parameters, counts) and every
2x2 tile square that phi = 1/2 crosses, with its binary32 corners, in
ascending tile order. Then `pfb_cell --boundary-out` against the file the
reference's `cell_gh200` writes for the same command line: identical
header, frame steps and times, cell records and end record, and the same
squares per cell (the reference appends a cell's squares in warp arrival
order, so they are compared as sorted sets)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pfb200
from pfb200 import boundary as bf
from pfb200._abi import CLASSES

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell"
REF = ROOT / "oracle" / "_ref" / "cell_gh200"


def expected_squares(tile):
    ll, lr = tile[:-1, :-1], tile[:-1, 1:]
    ur, ul = tile[1:, 1:], tile[1:, :-1]
    inside = ll >= 0.5
    hit = ((lr >= 0.5) != inside) | ((ur >= 0.5) != inside) | ((ul >= 0.5) != inside)
    y, x = np.nonzero(hit)  # row-major: ascending tile order
    out = np.zeros(x.size, bf.SQUARE_DTYPE)
    out["xy"] = x.astype(np.uint32) | (y.astype(np.uint32) << 16)
    out["phi"] = np.stack([ll[y, x], lr[y, x], ur[y, x], ul[y, x]], axis=1)
    return out


def check_frame(fr, phi, cells, side):
    for i in range(cells.size):
        c = cells[i]
        want = expected_squares(phi[i])
        np.testing.assert_array_equal(fr.squares[i], want)
        m = fr.cells[i]
        _, _, tx0, ty0 = CLASSES[int(c["cls"])]
        assert m["id"] == c["global_id"] and m["squares"] == want.size
        assert m["origin_x"] == (c["gx0"] - tx0) % side and m["origin_y"] == (c["gy0"] - ty0) % side
        for key, v in (("gamma", c["gamma"]), ("mobility", c["M_pf"]), ("active_speed", c["v_A"]),
                       ("radius", c["R_tgt"])):
            assert m[key] == v, key
        x = c["gx0"] + c["Cx"] / c["V"]
        y = c["gy0"] + c["Cy"] / c["V"]
        np.testing.assert_allclose([m["cx"], m["cy"]], [x % side, y % side], rtol=1e-6)


def test_frames_match_the_field(tmp_path):
    p = pfb200.SimParams2D(num_cells=12, L=320, target_radius=12.0, seed=8, v_A=0.05)
    cx, cy = pfb200.palmieri_centres(12, 320, 24.0, 8)
    sim = pfb200.Sim2D(p, cx, cy)
    sim.advance(30)
    sim.boundary_open(tmp_path / "b.pfb", interval=9)
    states = []
    for _ in range(3):
        sim.sync()
        states.append((sim.step, sim.phi(), sim.cells()))
        sim.boundary_capture()
        sim.advance(9)
    sim.boundary_close()
    sim.close()
    b = bf.read(tmp_path / "b.pfb")
    assert (b.cells, b.side, b.tile_pitch, b.dt, b.tau, b.level, b.interval, b.codec) == \
        (12, 320, 288, 0.01, 1.0e4, 0.5, 9, 0)
    assert [f.step for f in b.frames] == [s for s, _, _ in states]
    assert b.end_frames == 3 and b.end_step == states[-1][0]
    for fr, (step, phi, cells) in zip(b.frames, states):
        assert fr.time == step * 0.01
        check_frame(fr, phi, cells, 320)


def test_recorder_refusals(tmp_path):
    p = pfb200.SimParams2D(num_cells=4, L=320, target_radius=12.0, seed=3)
    cx, cy = pfb200.palmieri_centres(4, 320, 24.0, 3)
    sim = pfb200.Sim2D(p, cx, cy)
    (tmp_path / "old.pfb").write_bytes(b"")
    with pytest.raises(RuntimeError):
        sim.boundary_open(tmp_path / "old.pfb", interval=5)  # a new file only
    with pytest.raises(RuntimeError):
        sim.boundary_open(tmp_path / "z.pfb", interval=5, compress=True)  # no zstd here
    with pytest.raises(RuntimeError):
        sim.boundary_open(tmp_path / "i.pfb", interval=0)
    with pytest.raises(RuntimeError):
        sim.boundary_capture()  # nothing open
    sim.close()


ARGS = ("--N", 8, "--radius", 12, "--rho", 0.03, "--seed", 5, "--v-A", 0.05,
        "--trajectory-interval", 5, "--print-interval", 0, "--t-end", 0.23,
        "--boundary-interval", 7)


def run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
def test_cli_boundary_file_matches_reference(tmp_path):
    for who, exe in (("ours", EXE), ("theirs", REF)):
        d = tmp_path / who
        d.mkdir()
        run(exe, *ARGS, "--out", d / "traj.txt", "--boundary-out", d / "b.pfb")
    pa, pb = tmp_path / "ours" / "b.pfb", tmp_path / "theirs" / "b.pfb"
    assert pa.read_bytes()[:72] == pb.read_bytes()[:72]
    a, b = bf.read(pa), bf.read(pb)
    assert [f.step for f in a.frames] == [f.step for f in b.frames] == [0, 7, 14, 21, 23]
    assert [f.time for f in a.frames] == [f.time for f in b.frames]
    assert (a.end_step, a.end_time, a.end_frames) == (b.end_step, b.end_time, b.end_frames)
    for fa, fb in zip(a.frames, b.frames):
        assert fa.cells.tobytes() == fb.cells.tobytes()
        for sa, sb in zip(fa.squares, fb.squares):
            assert sa.tobytes() == np.sort(sb, order="xy").tobytes()
