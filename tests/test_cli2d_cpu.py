"""pfb_cell (the 2D command line) without a GPU: options, refusals and exit
codes (reference src/main.cu:340-560)."""
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
