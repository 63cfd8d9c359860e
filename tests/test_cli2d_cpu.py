"""pfb_cell (the 2D command line) without a GPU: options, refusals and exit
codes (reference src/main.cu:340-560)."""
import re
import subprocess
from pathlib import Path

import pytest

EXE = Path(__file__).resolve().parents[1] / "phase-field-gh200_b200" / "pfb200" / "_lib" / "pfb_cell"

pytestmark = pytest.mark.skipif(not EXE.exists(), reason="pfb_cell not built")


def run(*args):
    return subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True, timeout=60)


def test_help_lists_the_reference_options():
    r = run("--help")
    assert r.returncode == 0
    for opt in ("--N", "--radius", "--rho", "--v-A", "--t-end", "--checkpoint-dir",
                "--trajectory-interval", "--out", "--bench", "--velocity-moments",
                "--velocity-spatial-stride", "--velocity-dense-start",
                "--velocity-moments-reference", "--boundary-out", "--boundary-interval",
                "--boundary-compression"):
        assert opt in r.stdout


@pytest.mark.parametrize("args,code", [
    (("--bogus",), 2),
    (("--N",), 2),
    (("--N", "x"), 2),
    (("--dt", "nan"), 2),
    (("--velocity-moments", "v.bin"), 2),  # needs --out
    (("--velocity-moments", "v.bin", "--out", "v.bin"), 2),  # distinct paths
    (("--velocity-moments", "v.bin", "--out", "t.txt", "--velocity-spatial-stride", 0), 2),
    (("--velocity-moments", "v.bin", "--out", "t.txt", "--velocity-spatial-stride", 1001), 2),
    (("--velocity-moments", "v.bin", "--out", "t.txt", "--velocity-dense-start", -1), 2),
    (("--velocity-moments-reference",), 2),
    (("--velocity-moments", "v.bin", "--bench", 10), 2),
    (("--boundary-out", "b.bin"), 2),  # needs an interval
    (("--boundary-interval", 5), 2),  # needs a path
    (("--boundary-out", "b.bin", "--boundary-interval", 0), 2),
    (("--boundary-out", "b.bin", "--boundary-interval", 5, "--boundary-compression", "gz"), 2),
    (("--boundary-compression", "zstd"), 2),
    (("--boundary-out", "b.bin", "--boundary-interval", 5, "--bench", 10), 2),
    (("--boundary-out", "b.bin", "--boundary-interval", 5, "--out", "b.bin"), 2),
    (("--initial-centres", ""), 2),
])
def test_bad_options_exit_2(args, code):
    assert run(*args).returncode == code


def test_resume_refuses_domain_and_model_overrides(tmp_path):
    missing = tmp_path / "none.bin"
    assert run("-c", missing, "--N", 8).returncode == 2
    assert run("-c", missing, "--kappa", 3).returncode == 2
    r = run("-c", missing)
    assert r.returncode == 8 and "cannot open" in r.stderr


@pytest.mark.parametrize("text,ok", [
    ("1 0.25\n3 1.0\n", True),
    ("# comment\n\n  2\t0.75  \n", True),
    ("x 0.5\n", False),           # malformed id
    ("-1 0.5\n", False),          # negative id
    ("1 0.5 extra\n", False),     # trailing characters
    ("1 0\n", False),             # not positive
    ("1 1e39\n", False),          # not finite as binary32
    ("1 0.5\n1 0.6\n", False),    # duplicate id
    ("# only a comment\n", False),
    ("1\n", False),               # no value
])
def test_mobility_map_rules(tmp_path, text, ok):
    """Map files the reference refuses exit with status 2 before any device
    work; accepted ones get past reading (and then stop here, without a GPU,
    at initialisation)."""
    path = tmp_path / "m.txt"
    path.write_text(text)
    r = run("--N", 8, "--radius", 12, "--rho", 0.03, "--t-end", 0.01, "--phase-field-mobility-map", path)
    if ok:
        assert r.returncode != 2, r.stderr
    else:
        assert r.returncode == 2 and "mobility map" in r.stderr, r.stderr


SELF_TEST_ARGS = ("--self-test", "--N", 16, "--rho", 0.02, "--t-end", 0.01)


def self_test_numbers(text):
    """Ix of each separation and the Philox tau_eff printed by a self-test."""
    ix = [float(v) for v in re.findall(r"repulsive sign at separation \d+: Ix = (\S+)", text)]
    tau = re.search(r"Philox \w+: 5000000 (?:draws )?at p = \S+, tau_eff = (\S+)", text)
    return ix, float(tau.group(1)) if tau else None


def test_self_test_passes_and_matches_reference():
    r = subprocess.run([str(EXE), *map(str, SELF_TEST_ARGS)], capture_output=True, text=True, timeout=120)
    assert "--- self-test passed ---" in r.stdout and "[FAIL]" not in r.stdout, r.stdout
    ix, tau = self_test_numbers(r.stdout)
    assert len(ix) == 4 and all(v < 0 for v in ix) and tau is not None
    ref = EXE.parents[3] / "oracle" / "_ref" / "cell_gh200"
    if ref.exists():  # the reference prints its checks before it needs a device
        t = subprocess.run([str(ref), *map(str, SELF_TEST_ARGS)], capture_output=True, text=True, timeout=120)
        rix, rtau = self_test_numbers(t.stdout)
        assert rix == ix and rtau == tau


def test_self_test_failure_exits_4():
    # windows too small for the interface of a radius-110 cell
    r = subprocess.run([str(EXE), *map(str, SELF_TEST_ARGS), "--radius", "110"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 4 and "SELF-TEST FAILED" in r.stdout


@pytest.mark.parametrize("resume", [False, True])
def test_mobility_map_breaking_the_euler_bound_is_fatal(tmp_path, resume):
    """A map whose resolved (M_i/M0) gamma_i breaks dt * . * 40/6 < 1 stops the
    run before any device work, with the reference's message and its exit
    code (the reference's Sim::init fails: src/sim.cu:316, src/main.cu:611-615)."""
    import gzip
    m = tmp_path / "mob.txt"
    m.write_text("# one stiff cell\n0 100.0\n")
    if resume:
        ck = tmp_path / "ck.bin"
        src = Path(__file__).resolve().parent / "golden" / "ckpt2d_ref_n2.bin.gz"
        ck.write_bytes(gzip.decompress(src.read_bytes()))
        r = run("-c", ck, "--phase-field-mobility-map", m)
    else:
        r = run("--N", 12, "--phase-field-mobility-map", m)
    assert r.returncode == 5, r.stderr
    assert "[fatal] max_i[(M_i/M0)*gamma_i] = 200 gives dt*coeff*laplacian_bound" in r.stderr
    # an acceptable map passes the check (and then needs a device)
    m.write_text("0 0.6\n")
    r = run(*(("-c", tmp_path / "ck.bin") if resume else ("--N", 12)),
            "--phase-field-mobility-map", m)
    assert "laplacian_bound" not in r.stderr
