"""The bench's reference arm runs the oracle alone: it builds the workload
with the oracle's restatement of the reference's initialiser and loads no
library of this package, and it prints the same workload description as the
GPU arm."""
import json
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parent.parent

PROBE = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3"]
sys.path.insert(0, %r)
import bench
bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({"pfb_loaded": "libpfb200" in maps, "oracle_loaded": "liboracle2d" in maps}))
"""


def test_reference_arm_loads_only_the_oracle():
    out = subprocess.run([sys.executable, "-c", PROBE % str(REPO)], capture_output=True,
                         text=True, timeout=900, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    line, probe = lines[0], lines[-1]
    assert probe == {"pfb_loaded": False, "oracle_loaded": True}
    assert line["impl"] == "reference" and line["value"] > 0
    import bench

    class A:
        gpus = 1
        workload = "c2"
    assert line["config"] == bench.c2_config(A, 1024 * 144 * 144)
