"""Velocity observers of the 2D step and the PFVMOM4 recorder.

As the reference's velocity_observer_test.cu:229-352 does: observed steps
(advection and spatial) leave phi and every cell field but the observer
accumulators bit-identical to unobserved steps, and one observed step
agrees with the independent dense observer to 2e-9 (active, interaction,
interfacial, overlap and advection-correction channels). Then the recorder's
sampling schedule and file rules, and the PFVMOM4 file of
`pfb_cell --velocity-moments` against the one the reference's `cell_gh200`
writes for the same command line (fused and dense-reference modes)."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pfb200
from pfb200 import velocity as vf

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell"
REF = ROOT / "oracle" / "_ref" / "cell_gh200"
Q = slice(9, 21)  # the twelve integral channels


def make_sim(steps=40):
    """Twelve cells in a 320^2 box, frequent tumbles, 40 steps in."""
    p = pfb200.SimParams2D(num_cells=12, L=320, target_radius=12.0, seed=8, v_A=0.05, tau=2.0)
    cx, cy = pfb200.palmieri_centres(12, 320, 24.0, 8)
    sim = pfb200.Sim2D(p, cx, cy)
    sim.advance(steps)
    sim.sync()
    return sim


def without_accumulators(cells):
    c = cells.copy()
    c["adv_q"] = 0.0
    c["adv_count"] = 0
    return c.tobytes()


def test_observed_steps_leave_the_state_unchanged(tmp_path):
    plain, seen = make_sim(), make_sim()
    # stride 3 after two dense steps: a mix of spatial and advection steps
    seen.velocity_open(tmp_path / "v.bin", spatial_stride=3, dense_start=2)
    plain.advance(13)
    seen.advance(13)
    assert plain.phi().tobytes() == seen.phi().tobytes()
    assert without_accumulators(plain.cells()) == without_accumulators(seen.cells())
    assert np.all(seen.cells()["adv_count"] == 13)
    seen.velocity_close()
    plain.close()
    seen.close()


def record(tmp_path, name, steps, **kw):
    sim = make_sim()
    sim.velocity_open(tmp_path / name, **kw)
    sim.advance(steps)
    sim.velocity_capture()
    sim.velocity_close()
    sim.close()
    return vf.read(tmp_path / name)


def test_one_spatial_step_matches_the_dense_observer(tmp_path):
    fused = record(tmp_path, "f.bin", 1, spatial_stride=1, dense_start=10)
    dense = record(tmp_path, "d.bin", 1, reference=True)
    a, b = fused.rows[1], dense.rows[1]
    np.testing.assert_array_equal(a[:, :9], b[:, :9])  # ids, geometry, count
    np.testing.assert_allclose(a[:, Q], b[:, Q], rtol=0, atol=2e-9)
    assert np.all(a[:, 21] == 1)


def test_advection_steps_match_the_dense_observer(tmp_path):
    # the first step is always spatial; the second (step 41) is advection only
    fused = record(tmp_path, "f.bin", 2, spatial_stride=1000, dense_start=0)
    dense = record(tmp_path, "d.bin", 2, reference=True)
    a, b = fused.rows[1], dense.rows[1]
    np.testing.assert_allclose(a[:, 9:13], b[:, 9:13], rtol=0, atol=2e-9)
    assert np.all(a[:, 8] == 2) and np.all(a[:, 21] == 1)


@pytest.mark.parametrize("stride,dense", [(3, 0), (4, 5), (1, 0), (7, 2)])
def test_sampling_schedule(tmp_path, stride, dense):
    """Spatial samples: the first step after the open, the `dense` steps
    that follow the open, and steps that are multiples of the stride."""
    sim = make_sim()
    start = sim.step
    sim.velocity_open(tmp_path / "v.bin", spatial_stride=stride, dense_start=dense)
    for _ in range(4):
        sim.advance(5)
        sim.velocity_capture()
    sim.velocity_close()
    sim.close()
    f = vf.read(tmp_path / "v.bin")
    assert (f.start_step, f.spatial_stride, f.dense_start) == (start, stride, dense)
    np.testing.assert_array_equal(f.steps, start + np.arange(5) * 5)
    for k, step in enumerate(f.steps):
        expect = sum(1 for t in range(start, step)
                     if t == start or t < start + dense or t % stride == 0)
        assert np.all(f.rows[k, :, 8] == step - start)
        assert np.all(f.rows[k, :, 21] == expect), (k, stride, dense)


def test_recorder_file_rules(tmp_path):
    sim = make_sim(steps=2)
    path = tmp_path / "v.bin"
    path.write_bytes(b"")
    with pytest.raises(RuntimeError):
        sim.velocity_open(path)  # a new file only
    with pytest.raises(RuntimeError):
        sim.velocity_open(tmp_path / "w.bin", spatial_stride=0)
    sim.velocity_open(tmp_path / "w.bin", spatial_stride=5)
    with pytest.raises(RuntimeError):
        sim.velocity_open(tmp_path / "x.bin")  # one recorder at a time
    with pytest.raises(RuntimeError):
        sim.velocity_capture()  # no new step since the last frame
    sim.velocity_close()
    sim.close()


ARGS = ("--N", 8, "--radius", 12, "--rho", 0.03, "--seed", 5, "--v-A", 0.05, "--tau", 2,
        "--trajectory-interval", 5, "--print-interval", 0, "--t-end", 0.22)


def run(exe, *args):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]


def same_file(a, b):
    assert (a.cells, a.dt, a.start_step, a.side, a.spatial_stride, a.quadrature,
            a.dense_start) == (b.cells, b.dt, b.start_step, b.side, b.spatial_stride,
                               b.quadrature, b.dense_start)
    np.testing.assert_array_equal(a.steps, b.steps)
    ra, rb = a.rows, b.rows
    # id, counts exact; geometry and parameters from the same binary32 state
    for col in (0, 3, 4, 5, 6, 8, 21):
        np.testing.assert_array_equal(ra[..., col], rb[..., col], err_msg=str(col))
    np.testing.assert_allclose(ra[..., 1:3], rb[..., 1:3], rtol=0, atol=1e-9)
    np.testing.assert_allclose(ra[..., 7], rb[..., 7], rtol=1e-12)
    # integrals and rates: FP64 sums grouped differently (cluster bands
    # against one block), relative to each channel's scale; the area
    # channels (17, 18) are zero in exact arithmetic and hold roundoff only,
    # hence the absolute floor
    for col in list(range(9, 21)) + list(range(22, 26)):
        scale = np.abs(rb[..., col]).max()
        np.testing.assert_allclose(ra[..., col], rb[..., col], rtol=0,
                                   atol=max(1e-9 * scale, 1e-14), err_msg=str(col))


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
@pytest.mark.parametrize("mode", ["fused", "reference"])
def test_cli_velocity_file_matches_reference(tmp_path, mode):
    extra = (("--velocity-spatial-stride", 3, "--velocity-dense-start", 4) if mode == "fused"
             else ("--velocity-moments-reference",))
    for who, exe in (("ours", EXE), ("theirs", REF)):
        d = tmp_path / who
        d.mkdir()
        run(exe, *ARGS, *extra, "--out", d / "traj.txt", "--velocity-moments", d / "v.bin")
    a, b = vf.read(tmp_path / "ours" / "v.bin"), vf.read(tmp_path / "theirs" / "v.bin")
    np.testing.assert_array_equal(a.steps, [0, 5, 10, 15, 20, 22])
    same_file(a, b)
    head = (tmp_path / "ours" / "v.bin").read_bytes()[:56]
    assert head == (tmp_path / "theirs" / "v.bin").read_bytes()[:56]
