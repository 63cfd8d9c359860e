"""Adaptive 3D bricks on a B200: a cell whose support reaches its brick face
grows into a larger cube, promoted cubes are stepped, checkpointed and
cropped back. Checked against the reference's own cell_gh200_3d
(oracle/_ref) on the fixtures of its growth and promotion smoke runs
(reference tests/3d/run_two_gpu_growth_smoke.py,
tests/3d/run_promoted_regroup_smoke.py): a B=24 channel whose bricks get
planted tails that diffuse across the support margin, and a slab checkpoint
whose bricks are padded into larger cubes with exact zeros."""
import math
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pfb200
from pfb200 import boundary as bf
from pfb200 import checkpoint as ck

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell_3d"
REF = ROOT / "oracle" / "_ref" / "cell_gh200_3d"
needs_ref = pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")

DT = 0.001
POSITIONS = ((48, 48), (48, 42), (50, 24), (50, 72))
RHO = 4 * (4 * math.pi * 5 ** 3 / 3) / (10 * 95.5 ** 2)


def channel_args(centres):
    return ("--geometry", "channel", "--N", 4, "--radius", 5, "--lambda", 1,
            "--channel-height", 10, "--wall-padding", 3, "--wall-kappa", 10, "--wall-width", 1,
            "--rho", repr(RHO), "--brick-edge", 24, "--dt", DT, "--aging-time", 0, "--tau", 0.02,
            "--v-A", 0.1, "--gamma-cancer", 0.35, "--cancer-fraction", 0.5, "--seed", 20260909,
            "--polarity-seed", 20260910, "--initial-centres", centres, "--full-moment", 10,
            "--verify-every", 10)


def run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r


def rows(path):
    lines = Path(path).read_text().splitlines()
    return lines[:2], np.array([[float(v) for v in ln.split()] for ln in lines[2:]])


def centres_table(tmp_path):
    c = tmp_path / "centres.csv"
    c.write_text("global_id,x,y,z\n" + "".join(f"{g},{x},{y},5\n" for g, (x, y) in enumerate(POSITIONS)))
    return c


def plant_tails(src, dst, ids):
    """The reference growth fixture: phi = 0.25 at x in {4, 19}, y and z in
    {11, 12} of each listed B=24 brick; the tails diffuse across the support
    margin during the next steps."""
    got = ck.read3d(src)
    packed = got.packed.copy()
    fields = []
    off = 0
    for e in got.edges():
        fields.append(packed[off:off + e ** 3].reshape(e, e, e))
        off += e ** 3
    for n in ids:
        assert got.edges()[n] == 24
        for z in (11, 12):
            for y in (11, 12):
                for x in (4, 19):
                    fields[n][z, y, x] = 0.25
    ck.write3d(dst, got.params, got.step, got.cells, packed, got.base_measure_shards)


def pad_cubes(src, dst, ids, pad=4):
    """The reference promotion fixture: each listed brick embedded in a cube
    `2 pad` wider with exact zeros, origin moved by -pad, centroid sums by
    pad V, support box by +pad (world field unchanged)."""
    got = ck.read3d(src)
    cells = got.cells.copy()
    out = []
    for n, f in enumerate(got.fields()):
        if n not in ids:
            out.append(f.ravel())
            continue
        e = f.shape[0] + 2 * pad
        cube = np.zeros((e, e, e), np.float32)
        cube[pad:pad + f.shape[0], pad:pad + f.shape[0], pad:pad + f.shape[0]] = f
        for k in "xyz":
            cells["origin_" + k][n] -= pad
            cells["C" + k][n] += pad * cells["V"][n]
            cells["bb_lo_" + k][n] += pad
            cells["bb_hi_" + k][n] += pad
        cells["storage_edge"][n] = e
        out.append(cube.ravel())
    ck.write3d(dst, got.params, got.step, cells, np.concatenate(out), got.base_measure_shards)


def world_fields(c3d):
    return c3d.fields(), c3d.edges()


def same_state(a, b, tol=1e-5):
    """Same step, storage edges, origins and counters; fields within tol."""
    assert a.step == b.step
    assert bytes(a.params) == bytes(b.params)
    np.testing.assert_array_equal(a.edges(), b.edges())
    for f in ("global_id", "origin_x", "origin_y", "origin_z", "shift_ctr", "tumble_ctr",
              "storage_edge"):
        np.testing.assert_array_equal(a.cells[f], b.cells[f], err_msg=f)
    for fa, fb in zip(a.fields(), b.fields()):
        np.testing.assert_allclose(fa, fb, rtol=0, atol=tol)


def same_boundary(pa, pb):
    """PFB3D files of the two programs: same header, frame steps, per-cell
    records (cube edges included) and squares (corner values to 1e-5; a
    square present in one file only has a corner at the 0.5 level)."""
    assert pa.read_bytes()[:128] == pb.read_bytes()[:128]
    a, b = bf.read3d(pa), bf.read3d(pb)
    assert a.complete and b.complete
    assert [f.step for f in a.frames] == [f.step for f in b.frames]
    edges = []
    for fa, fb in zip(a.frames, b.frames):
        for k in ("id", "origin_x", "origin_y", "origin_z", "brick_edge", "plane_edge"):
            np.testing.assert_array_equal(fa.cells[k], fb.cells[k], err_msg=k)
        edges.append(np.asarray(fa.cells["brick_edge"]).max())
        for sa, sb in zip(fa.squares, fb.squares):
            ka, kb = dict(zip(sa["xy"], sa["phi"])), dict(zip(sb["xy"], sb["phi"]))
            for xy in set(ka) & set(kb):
                np.testing.assert_allclose(ka[xy], kb[xy], rtol=0, atol=1e-5)
            for xy in set(ka) ^ set(kb):
                corners = ka.get(xy, kb.get(xy))
                assert np.min(np.abs(corners - 0.5)) < 2e-5, (hex(xy), corners)
    return edges


def same_rows(a, b):
    assert a.shape == b.shape
    np.testing.assert_array_equal(a[:, :2], b[:, :2])
    np.testing.assert_allclose(a[:, 2:5], b[:, 2:5], rtol=0, atol=1e-8)
    np.testing.assert_allclose(a[:, 5:], b[:, 5:], rtol=1e-6, atol=1e-8)


@needs_ref
@pytest.mark.parametrize("ids", [(1,), (0, 1)], ids=["one", "two"])
def test_runtime_growth_matches_reference(tmp_path, ids):
    """Resumed from the planted fixture, both programs grow the same cells
    from B=24 to the next tier during the same steps and reach the same state
    40 steps in; the rows and the final checkpoints agree."""
    centres = centres_table(tmp_path)
    src = tmp_path / "src"
    run(REF, *channel_args(centres), "--t-end", 10 * DT, "--print-interval", 0,
        "--checkpoint-dir", src)
    fixture = tmp_path / "fixture.pf3d"
    plant_tails(src / "checkpoint.pf3d", fixture, ids)
    outs = {}
    for name, exe in (("ours", EXE), ("theirs", REF)):
        d = tmp_path / name
        r = run(exe, "-c", fixture, "--t-end", 40 * DT, "--print-interval", 0,
                "--trajectory-interval", 10, "--out", d / "traj.txt", "--checkpoint-dir", d,
                "--boundary-out", d / "b.pfb3d", "--boundary-interval", 10,
                "--boundary-projection", "maximum")
        outs[name] = (ck.read3d(d / "checkpoint.pf3d"), rows(d / "traj.txt"), r.stdout)
    a, b = outs["ours"][0], outs["theirs"][0]
    assert "[3d] resized" in outs["theirs"][2]
    grown = [n for n, e in enumerate(b.edges()) if e > 24]
    assert sorted(grown) == sorted(ids)
    same_state(a, b)
    (ha, ra), (hb, rb) = outs["ours"][1], outs["theirs"][1]
    assert ha == hb
    same_rows(ra, rb)
    edges = same_boundary(tmp_path / "ours" / "b.pfb3d", tmp_path / "theirs" / "b.pfb3d")
    assert edges[0] == 24 and edges[-1] > 24  # frames before and after the growth


@needs_ref
def test_promoted_checkpoint_resume_matches_reference(tmp_path):
    """A checkpoint whose cells 0 and 2 sit on 32^3 cubes (B=24 bricks padded
    with zeros): both programs resume it, step the promoted cubes for 41
    steps and write the same state; each resumes the other's result."""
    centres = centres_table(tmp_path)
    src = tmp_path / "src"
    run(REF, *channel_args(centres), "--t-end", 10 * DT, "--print-interval", 0,
        "--checkpoint-dir", src)
    fixture = tmp_path / "padded.pf3d"
    pad_cubes(src / "checkpoint.pf3d", fixture, (0, 2))
    res = {}
    for name, exe in (("ours", EXE), ("theirs", REF)):
        d = tmp_path / name
        run(exe, "-c", fixture, "--t-end", 51 * DT, "--print-interval", 0,
            "--trajectory-interval", 1, "--out", d / "traj.txt", "--checkpoint-dir", d)
        res[name] = ck.read3d(d / "checkpoint.pf3d")
    a, b = res["ours"], res["theirs"]
    assert (b.edges()[[0, 2]] >= 32).all()
    same_state(a, b)
    _, ra = rows(tmp_path / "ours" / "traj.txt")
    _, rb = rows(tmp_path / "theirs" / "traj.txt")
    same_rows(ra, rb)
    # each continues the other's promoted state
    run(EXE, "-c", tmp_path / "theirs" / "checkpoint.pf3d", "--t-end", 61 * DT, "--print-interval", 0,
        "--checkpoint-dir", tmp_path / "ours2")
    run(REF, "-c", tmp_path / "ours" / "checkpoint.pf3d", "--t-end", 61 * DT, "--print-interval", 0,
        "--checkpoint-dir", tmp_path / "theirs2")
    same_state(ck.read3d(tmp_path / "ours2" / "checkpoint.pf3d"),
               ck.read3d(tmp_path / "theirs2" / "checkpoint.pf3d"))


def test_compaction_crops_a_padded_cube(tmp_path):
    """Cell 1 of a fresh state padded from B = 24 into a 56^3 cube, restarted
    at step 1023: the step to 1024 ends with a compaction, which crops the
    cube to 48 (16 spare planes beyond the support on every face; the shell
    outside the retained cube's 8-plane guard band holds exact zeros). Its
    world field equals that of the same step without the padding."""
    p = pfb200.SimParams3D(Nx=96, Ny=96, Nz=96, geometry="periodic", num_cells=2, target_radius=5.0,
                           lambda_=1.0, B=24, seed=3, v_A=0.0, full_moment_every=0)
    # off the half-voxel ties of integer centres, so both runs plan the same shifts
    c = np.array([[30.3, 40.2, 50.1], [70.2, 60.35, 30.15]])
    s = pfb200.Sim3D(p, c)
    cells, packed = s.cells(), s.packed()
    s.close()
    src = tmp_path / "base.pf3d"
    ck.write3d(src, ck.params_record3d(p, 24), 1023, cells, packed, 4)
    padded = tmp_path / "padded.pf3d"
    pad_cubes(src, padded, (1,), pad=16)
    ref = ck.restart3d(src)
    big = ck.restart3d(padded)
    assert big.promoted_count == 1 and big.cells()["storage_edge"][1] == 56
    for sim in (ref, big):
        sim.advance(1)
        assert sim.step == 1024
    cb = big.cells()
    assert cb["storage_edge"][1] == 48 and big.promoted_count == 1
    ca = ref.cells()
    fa, fb = ref.fields(), big.fields()
    np.testing.assert_array_equal(fa[0], fb[0])
    # the 48^3 cube holds the 24^3 brick 12 planes in, zeros around it
    for k in "xyz":
        assert cb["origin_" + k][1] == ca["origin_" + k][1] - 12
    np.testing.assert_allclose(fb[1][12:36, 12:36, 12:36], fa[1], rtol=0, atol=1e-6)
    inner = np.zeros((48, 48, 48), bool)
    inner[12:36, 12:36, 12:36] = True
    assert not fb[1][~inner].any()
    ref.close()
    big.close()
