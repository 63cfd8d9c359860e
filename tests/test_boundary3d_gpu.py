"""PFB3D boundary recorder of the 3D system (reference
src/pf3d/boundary_output.cu).

Each frame is checked against a numpy restatement on the same state, for
the maximum projection in all three geometries and the basal projection on
the slab: every cell's (B+2)^2 plane is the maximum of its brick over the
in-domain z planes (or the substrate plane), with a zero ring; the cell
records and the crossed squares with their binary32 corners in ascending
plane order must match exactly. Then `pfb_cell_3d --boundary-out` against
the reference's `cell_gh200_3d` on the same command line: identical header,
frame steps and times, end record and cell records; squares within the 3D
field tolerance (1e-5 on phi), a square present in one file only allowed
where a corner lies that close to the level."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pfb200
from pfb200 import boundary as bf

from helpers3d import small_centres, small_params

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell_3d"
REF = ROOT / "oracle" / "_ref" / "cell_gh200_3d"


def projected(brick, oz, nz, periodic, basal):
    B = brick.shape[0]
    if basal:
        z0, z1 = (-oz, -oz + 1) if -B < oz <= 0 else (0, 0)
    elif periodic:
        z0, z1 = 0, B
    elif oz >= nz or oz <= -B:
        z0, z1 = 0, 0
    else:
        z0, z1 = max(0, -oz), min(B, nz - oz)
    plane = np.zeros((B + 2, B + 2), np.float32)
    if z0 < z1:
        plane[1:-1, 1:-1] = brick[z0:z1].max(axis=0)
    return plane


def crossed(plane):
    ll, lr = plane[:-1, :-1], plane[:-1, 1:]
    ur, ul = plane[1:, 1:], plane[1:, :-1]
    inside = ll >= 0.5
    hit = ((lr >= 0.5) != inside) | ((ur >= 0.5) != inside) | ((ul >= 0.5) != inside)
    y, x = np.nonzero(hit)
    out = np.zeros(x.size, bf.SQUARE_DTYPE)
    out["xy"] = x.astype(np.uint32) | (y.astype(np.uint32) << 16)
    out["phi"] = np.stack([ll[y, x], lr[y, x], ur[y, x], ul[y, x]], axis=1)
    return out


@pytest.mark.parametrize("geometry,projection", [("periodic", "maximum"), ("slab", "maximum"),
                                                 ("slab", "basal"), ("channel", "maximum")])
def test_frames_match_the_projection(tmp_path, geometry, projection):
    p = small_params(geometry)
    sim = pfb200.Sim3D(p, small_centres(p))
    sim.advance(2)
    sim.boundary_open(tmp_path / "b.pfb3d", interval=3, projection=projection)
    states = []
    for _ in range(3):
        sim.sync()
        states.append((sim.step, sim.phi(), sim.cells()))
        sim.boundary_capture()
        sim.advance(3)
    sim.boundary_close()
    B = sim.B
    sim.close()
    b = bf.read3d(tmp_path / "b.pfb3d")
    assert b.complete and b.cells == p.num_cells and b.shape == (p.Nx, p.Ny, p.Nz)
    assert b.projection == {"basal": 1, "maximum": 2}[projection] and b.interval == 3
    assert [f.step for f in b.frames] == [s for s, _, _ in states]
    assert b.end_step == states[-1][0]
    for fr, (step, phi, cells) in zip(b.frames, states):
        assert fr.time == step * p.dt
        for i in range(p.num_cells):
            c, m = cells[i], fr.cells[i]
            assert (m["id"], m["origin_x"], m["origin_y"], m["origin_z"]) == \
                (c["global_id"], c["origin_x"] - 1, c["origin_y"] - 1, c["origin_z"])
            assert (m["brick_edge"], m["plane_edge"]) == (B, B + 2)
            assert (m["gamma"], m["active_speed"], m["radius"]) == (c["gamma"], c["v_A"], c["R_tgt"])
            want = crossed(projected(phi[i], int(c["origin_z"]), p.Nz, geometry == "periodic",
                                     projection == "basal"))
            assert m["squares"] == want.size
            np.testing.assert_array_equal(fr.squares[i], want)


def test_recorder_refusals(tmp_path):
    p = small_params("periodic")
    sim = pfb200.Sim3D(p, small_centres(p))
    (tmp_path / "old").write_bytes(b"")
    for kw in (dict(path=tmp_path / "old"), dict(projection="basal"), dict(compress=True),
               dict(interval=0)):
        args = dict(path=tmp_path / "new", interval=2, projection="maximum", compress=False)
        args.update(kw)
        with pytest.raises(RuntimeError):
            sim.boundary_open(args.pop("path"), **args)
    sim.boundary_open(tmp_path / "a", interval=2)
    sim.boundary_capture()
    with pytest.raises(RuntimeError):
        sim.boundary_capture()  # the same step twice
    sim.close()  # an unfinished recording stays unterminated
    b = bf.read3d(tmp_path / "a")
    assert not b.complete and len(b.frames) == 1


ARGS = ("--N", 3, "--radius", 4, "--lambda", 3, "--v-A", 0.05, "--seed", 11,
        "--print-interval", 0, "--t-end", 0.05, "--boundary-interval", 2)


def run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
@pytest.mark.parametrize("geometry,rho,projection", [("periodic", 0.007, "maximum"),
                                                     ("slab", 0.05, "basal"),
                                                     ("slab", 0.05, "maximum")])
def test_cli_boundary_file_matches_reference(tmp_path, geometry, rho, projection):
    for who, exe in (("ours", EXE), ("theirs", REF)):
        d = tmp_path / who
        d.mkdir()
        run(exe, *ARGS, "--geometry", geometry, "--rho", rho, "--boundary-projection", projection,
            "--boundary-out", d / "b.pfb3d")
    pa, pb = tmp_path / "ours" / "b.pfb3d", tmp_path / "theirs" / "b.pfb3d"
    assert pa.read_bytes()[:128] == pb.read_bytes()[:128]
    a, b = bf.read3d(pa), bf.read3d(pb)
    assert a.complete and b.complete
    assert [f.step for f in a.frames] == [f.step for f in b.frames] == [0, 2, 4, 5]
    assert [f.time for f in a.frames] == [f.time for f in b.frames]
    assert (a.end_step, a.end_time) == (b.end_step, b.end_time)
    for fa, fb in zip(a.frames, b.frames):
        same = ["id", "origin_x", "origin_y", "origin_z", "brick_edge", "plane_edge", "gamma",
                "active_speed", "radius"]
        for k in same:
            np.testing.assert_array_equal(fa.cells[k], fb.cells[k], err_msg=k)
        for sa, sb in zip(fa.squares, fb.squares):
            ka, kb = dict(zip(sa["xy"], sa["phi"])), dict(zip(sb["xy"], sb["phi"]))
            for xy in set(ka) & set(kb):
                np.testing.assert_allclose(ka[xy], kb[xy], rtol=0, atol=1e-5)
            for xy in set(ka) ^ set(kb):
                corners = ka.get(xy, kb.get(xy))
                assert np.min(np.abs(corners - 0.5)) < 2e-5, (hex(xy), corners)
