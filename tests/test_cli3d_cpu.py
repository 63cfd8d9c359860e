"""pfb_cell_3d on the host: the reference's option ranges and usage errors
(exit status 2), the resume contract, and the fresh placement of every
geometry against the oracle's restatement (the program prints the centre
table's hash before it touches a device)."""
import math
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import placement as pl  # noqa: E402

EXE = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell_3d"
pytestmark = pytest.mark.skipif(not EXE.exists(), reason="pfb_cell_3d not built")


def run(*args):
    return subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True, timeout=120)


def test_mt19937_64_known_answer():
    g = pl.MT19937_64()
    for _ in range(9999):
        g()
    assert g() == 9981545732273789042


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libref3d_cpu.so").exists(),
                    reason="reference host build absent")
@pytest.mark.parametrize("seed", [1, 9, 1234])
def test_placements_pinned_to_reference(seed):
    import ctypes as C
    import oracle3d as o3
    L = o3.rclib()
    F = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    n = 8
    x, y, z = (np.zeros(n, np.float32) for _ in range(3))
    assert L.ref3d_cpu_palmieri3d(n, 40.0, 6.0, seed, F(x), F(y), F(z)) == 0
    a, b, c = pl.palmieri3d(n, 40.0, 6.0, seed)
    for u, v in ((x, a), (y, b), (z, c)):
        np.testing.assert_array_equal(u, v)
    assert L.ref3d_cpu_table_hash(n, F(x), F(y), F(z)) == pl.table_hash(a, b, c)
    assert L.ref3d_cpu_channel3d(n, 60.0, 13, 6.0, seed, F(x), F(y), F(z)) == 0
    a, b, c = pl.channel3d(n, 60.0, 13, 6.0, seed)
    for u, v in ((x, a), (y, b), (z, c)):
        np.testing.assert_array_equal(u, v)
    assert L.ref3d_cpu_palmieri2d(n, 90.0, 12.0, seed, F(x), F(y)) == 0
    a, b = pl.palmieri2d(n, 90.0, 12.0, seed)
    np.testing.assert_array_equal(x, a)
    np.testing.assert_array_equal(y, b)


def test_slab_placement_matches_library_2d_placement():
    import pfb200
    for seed in (1, 7, 1234):
        x, y = pl.palmieri2d(10, 150.0, 20.0, seed)
        a, b = pfb200.palmieri_centres(10, 150, 20.0, seed)
        np.testing.assert_array_equal(x, a)
        np.testing.assert_array_equal(y, b)


def test_help():
    r = run("--help")
    assert r.returncode == 0 and "--geometry" in r.stdout


@pytest.mark.parametrize("args,msg", [
    (("--rho", 1.5), "--rho expects"),
    (("--N", 0), "--N expects"),
    (("--radius", "abc"), "--radius expects"),
    (("--geometry", "torus"), "--geometry expects"),
    (("--slab-height", 40), "requires --geometry slab"),
    (("--channel-height", 40), "requires --geometry channel"),
    (("--geometry", "slab", "--wall-width", 2), "require --geometry channel"),
    (("--geometry", "slab", "--wall-padding", 9), "requires --geometry channel"),
    (("--geometry", "channel", "--radius", 8, "--channel-height", 10), "one-diameter minimum"),
    (("--geometry", "channel", "--lambda", 3, "--wall-padding", 5), "smaller than the minimum"),
    (("--geometry", "slab", "--radius", 8, "--lambda", 3, "--slab-height", 3), "must exceed"),
    (("--cancer-fraction", 1.5), "--cancer-fraction expects"),
    (("--memory-mode", "fast"), "--memory-mode expects"),
    (("--measure-shards", 8), "measures with --measure-shards 4 only"),
    (("--promoted-measure-shards", 4), "--promoted-measure-shards 0 only"),
    (("--scratch-slots", -2), "--scratch-slots expects"),
    (("--peer-device", 1), "unknown option"),
    (("--trajectory-interval", 0), "--trajectory-interval expects"),
    (("--seed", -4), "unsigned"),
    (("--out",), "requires a value"),
    (("--boundary-out", "b.pfb3d"), "requires --boundary-out and --boundary-interval"),
    (("--boundary-interval", 5), "requires --boundary-out and --boundary-interval"),
    (("--boundary-out", "b", "--boundary-interval", 5, "--boundary-projection", "flat"),
     "expects maximum or basal"),
    (("--boundary-out", "b", "--boundary-interval", 5, "--boundary-compression", "gz"),
     "expects none or zstd"),
    (("--boundary-out", "b", "--boundary-interval", 5, "--bench", 3), "cannot be combined"),
    (("--boundary-out", "b", "--boundary-interval", 5, "--boundary-projection", "basal"),
     "requires --geometry slab"),
])
def test_usage_errors(args, msg):
    r = run(*args)
    assert r.returncode == 2, r.stdout + r.stderr
    assert msg in r.stderr


def test_resume_keeps_the_checkpoint_model(tmp_path):
    r = run("-c", tmp_path / "missing.pf3d", "--N", 4)
    assert r.returncode == 2 and "preserves its model" in r.stderr
    r = run("-c", tmp_path / "missing.pf3d", "--t-end", 3)
    assert r.returncode == 1  # the file cannot be read


CASE = dict(N=6, radius=8.0, lam=3.0, rho=0.05, seed=9)


def printed_hash(geometry):
    c = CASE
    r = run("--geometry", geometry, "--N", c["N"], "--radius", c["radius"], "--lambda", c["lam"],
            "--rho", c["rho"], "--seed", c["seed"], "--t-end", 0.1, "--print-interval", 0)
    m = re.search(r"table hash ([0-9a-f]{16})", r.stdout)
    assert m, r.stdout + r.stderr
    return int(m.group(1), 16)


def test_periodic_placement_hash():
    c = CASE
    side, _, _, _ = pl.domain3d("periodic", c["N"], c["radius"], c["rho"], c["lam"])
    x, y, z = pl.palmieri3d(c["N"], float(side), c["radius"], c["seed"])
    assert printed_hash("periodic") == pl.table_hash(x, y, z)


def test_slab_placement_hash():
    c = CASE
    side, _, _, _ = pl.domain3d("slab", c["N"], c["radius"], c["rho"], c["lam"])
    x, y = pl.palmieri2d(c["N"], float(side), c["radius"], c["seed"])
    z = np.full_like(x, -0.5)
    assert printed_hash("slab") == pl.table_hash(x, y, z)


def test_channel_placement_hash():
    c = CASE
    side, _, H, _ = pl.domain3d("channel", c["N"], c["radius"], c["rho"], c["lam"])
    assert H == math.ceil(2 * c["radius"])
    x, y, z = pl.channel3d(c["N"], float(side), H, c["radius"], c["seed"])
    assert np.all((z >= c["radius"]) & (z <= H - c["radius"]))
    assert printed_hash("channel") == pl.table_hash(x, y, z)


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libref3d_cpu.so").exists(),
                    reason="reference host build absent")
@pytest.mark.parametrize("n,fraction,seed", [(3, 0.34, 11), (10, 0.5, 1234), (288, 0.1, 7),
                                             (97, 1.0, 3), (50, 0.0, 5), (1, 0.6, 9)])
def test_soft_identities_match_reference(n, fraction, seed):
    import ctypes as C
    import oracle3d as o3
    from pfb200._abi import lib
    theirs = np.zeros(n, np.uint8)
    ours = np.zeros(n, np.uint8)
    assert o3.rclib().ref_soft_membership(n, fraction, seed, theirs.ctypes.data) == 0
    assert lib().pfb3d_soft_membership(n, fraction, seed, ours.ctypes.data) == 0
    np.testing.assert_array_equal(ours, theirs)
    assert ours.sum() == round(fraction * n)
