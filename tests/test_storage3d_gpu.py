"""3D storage modes on a B200 (reference StorageMode3D, --memory-mode):
throughput (two phi pools, two aggregates), balanced (one pool, two
aggregates, scratch bricks) and compact (one pool, one aggregate rebuilt
after every update) give the same cells, fields, aggregate and flags, bit
for bit, in all three geometries, with fewer scratch bricks than cells (the
update then runs in batches), with promoted cubes, and across the 1024-step
compaction; the command line in compact mode matches the reference's."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pfb200
from pfb200 import checkpoint as ck
from helpers3d import small_centres, small_params

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell_3d"
REF = ROOT / "oracle" / "_ref" / "cell_gh200_3d"


def state(sim):
    return sim.cells(), sim.packed(), sim.S(), sim.flags()


def assert_same(a, b):
    assert a[0].tobytes() == b[0].tobytes()
    assert a[1].tobytes() == b[1].tobytes()
    assert a[2].tobytes() == b[2].tobytes()
    np.testing.assert_array_equal(a[3], b[3])


@pytest.mark.parametrize("geometry", ["periodic", "slab", "channel"])
def test_modes_are_bit_identical(geometry):
    p = small_params(geometry, full_moment_every=7)
    c = small_centres(p)
    out = {}
    for mode, slots in (("throughput", 0), ("balanced", 0), ("balanced", 4), ("compact", 5)):
        s = pfb200.Sim3D(p, c, memory_mode=mode, scratch_slots=slots)
        assert s.memory_mode == mode
        if mode != "throughput":
            assert s.scratch_slots == (slots or p.num_cells)
        s.advance(29)
        out[(mode, slots)] = state(s)
        s.close()
    ref = out[("throughput", 0)]
    for k, v in out.items():
        assert_same(ref, v)
    assert not ref[3].any()


def test_modes_with_promoted_cubes(tmp_path):
    """Two cells padded into 48^3 cubes (B = 40): the promoted cubes keep
    their double buffers in every mode; 12 steps agree bit for bit."""
    p = small_params("periodic", N=6)
    s = pfb200.Sim3D(p, small_centres(p))
    cells, packed = s.cells(), s.packed()
    s.close()
    src = tmp_path / "base.pf3d"
    ck.write3d(src, ck.params_record3d(p, 40), 0, cells, packed, 4)
    padded = tmp_path / "padded.pf3d"
    from test_adaptive3d_gpu import pad_cubes
    pad_cubes(src, padded, (1, 4), pad=4)
    out = []
    for mode in ("throughput", "balanced", "compact"):
        sim = ck.restart3d(padded, memory_mode=mode, scratch_slots=3 if mode != "throughput" else 0)
        assert sim.promoted_count == 2
        sim.advance(12)
        out.append(state(sim))
        sim.close()
    assert_same(out[0], out[1])
    assert_same(out[0], out[2])


@pytest.mark.skipif(not REF.exists(), reason="reference CLI not built")
@pytest.mark.parametrize("mode", ["balanced", "compact"])
def test_cli_memory_mode_matches_reference(tmp_path, mode):
    args = ("--N", 3, "--radius", 4, "--lambda", 3, "--v-A", 0.05, "--seed", 11, "--rho", 0.05,
            "--geometry", "slab", "--t-end", 0.03, "--trajectory-interval", 2, "--print-interval", 0,
            "--memory-mode", mode, "--scratch-slots", 2)
    for who, exe in (("ours", EXE), ("theirs", REF)):
        d = tmp_path / who
        r = subprocess.run([str(exe), *map(str, args), "--out", str(d / "traj.txt"),
                            "--checkpoint-dir", str(d)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    a, b = ck.read3d(tmp_path / "ours" / "checkpoint.pf3d"), ck.read3d(tmp_path / "theirs" / "checkpoint.pf3d")
    assert a.step == b.step == 3
    assert bytes(a.params) == bytes(b.params)
    np.testing.assert_allclose(a.packed, b.packed, rtol=0, atol=1e-5)
    la = (tmp_path / "ours" / "traj.txt").read_text().splitlines()
    lb = (tmp_path / "theirs" / "traj.txt").read_text().splitlines()
    assert la[:2] == lb[:2] and len(la) == len(lb)
