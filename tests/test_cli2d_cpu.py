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
