"""--initial-centres of pfb_cell and pfb_cell_3d against the reference's own
table readers (compiled from its headers into oracle/_ref/libref3d_cpu.so):
for every table format, a family of well-formed and malformed tables
(header, line ends, byte-order mark, field count, number syntax, id order,
row count, box, separation, centre cell, channel clearance, source_L) is
accepted or refused alike, and an accepted table gives the same centre-table
hash. The programs print the hash before touching a device, so this runs on
the host."""
import ctypes as C
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

LIB = ROOT / "phase-field-gh200_b200" / "pfb200" / "_lib"
REF_SO = ROOT / "oracle" / "_ref" / "libref3d_cpu.so"
pytestmark = pytest.mark.skipif(not REF_SO.exists() or not (LIB / "pfb_cell_3d").exists(),
                                reason="reference host build or command lines absent")


def ref():
    import oracle3d as o3
    return o3.rclib()


def fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def cli_hash(exe, args):
    r = subprocess.run([str(LIB / exe), *map(str, args)], capture_output=True, text=True, timeout=60)
    m = re.search(r"table hash ([0-9a-f]{16})", r.stdout)
    return int(m.group(1), 16) if m else None


def fmt(v):
    return repr(float(v)) if isinstance(v, float) else str(v)


def write(path, header, rows, eol="\n", bom=False, extra=()):
    lines = [header] + list(extra) + [",".join(fmt(v) for v in r) for r in rows]
    data = eol.join(lines) + eol
    path.write_bytes((b"\xef\xbb\xbf" if bom else b"") + data.encode())
    return path


# ---- 2D periodic table (pfb_cell) ------------------------------------------------
N2, R2, RHO2 = 4, 12.0, 0.02


def side2():
    import pfb200
    return pfb200.domain_side_for(N2, R2, RHO2)


def good2(L):
    c = L / 2
    return [[0, c, c], [1, 10.5, 20.25], [2, 200.0, 30.0], [3, 60.0, 250.5]]


def variants2(L):
    g = good2(L)
    yield "good", "global_id,x,y", g, {}
    yield "exp", "global_id,x,y", [g[0], [1, "1.05e1", "2.025e1"], g[2], g[3]], {}
    yield "crlf", "global_id,x,y", g, {"eol": "\r\n"}
    yield "bom", "global_id,x,y", g, {"bom": True}
    yield "header", "id,x,y", g, {}
    yield "order", "global_id,x,y", [g[0], g[2], g[1], g[3]], {}
    yield "short", "global_id,x,y", g[:3], {}
    yield "long", "global_id,x,y", g + [[4, 100.0, 100.0]], {}
    yield "box", "global_id,x,y", [g[0], [1, float(L), 20.0], g[2], g[3]], {}
    yield "close", "global_id,x,y", [g[0], [1, L / 2 + 11.9, L / 2], g[2], g[3]], {}
    yield "edge", "global_id,x,y", [g[0], [1, L / 2 + 12.0, L / 2], g[2], g[3]], {}
    yield "wrap", "global_id,x,y", [g[0], g[1], g[2], [3, L - 1.0, 20.0]], {}
    yield "centre", "global_id,x,y", [[0, L / 2 + 0.5, L / 2]] + g[1:], {}
    yield "syntax", "global_id,x,y", [g[0], [1, "10.5x", 20.0], g[2], g[3]], {}
    yield "space", "global_id,x,y", [g[0], [1, " 10.5", 20.0], g[2], g[3]], {}
    yield "nan", "global_id,x,y", [g[0], [1, "nan", 20.0], g[2], g[3]], {}
    yield "fields", "global_id,x,y", [g[0], [1, 10.5, 20.0, 1.0], g[2], g[3]], {}


@pytest.mark.parametrize("case", [v[0] for v in variants2(400)])
def test_table2_like_reference(tmp_path, case):
    L = side2()
    name, header, rows, kw = next(v for v in variants2(L) if v[0] == case)
    path = write(tmp_path / f"{name}.csv", header, rows, **kw)
    x, y = np.zeros(N2, np.float32), np.zeros(N2, np.float32)
    h = C.c_uint64()
    rc = ref().ref_read_table2(str(path).encode(), N2, float(L), R2, fptr(x), fptr(y), C.byref(h))
    ours = cli_hash("pfb_cell", ["--N", N2, "--radius", R2, "--rho", RHO2, "--t-end", 0.01,
                                 "--initial-centres", path])
    if rc == 0:
        assert ours == h.value, (case, ours, h.value)
    else:
        assert ours is None, case


# ---- 3D periodic table (pfb_cell_3d --geometry periodic) ----------------------------
N3, R3, LAM3 = 3, 4.0, 3.0


def side3(geometry, rho):
    return pl.domain3d(geometry, N3, R3, rho, LAM3)


def variants3(L):
    c = L / 2
    g = [[0, c, c, c], [1, 5.5, 6.25, 7.0], [2, 40.0, 40.5, 10.0]]
    yield "good", "global_id,x,y,z", g, {}
    yield "crlf", "global_id,x,y,z", g, {"eol": "\r\n"}
    yield "header", "global_id,x,y", g, {}
    yield "order", "global_id,x,y,z", [g[0], g[2], g[1]], {}
    yield "long", "global_id,x,y,z", g + [[3, 1.0, 1.0, 1.0]], {}
    yield "box", "global_id,x,y,z", [g[0], g[1], [2, 40.0, 40.5, float(L)]], {}
    yield "close", "global_id,x,y,z", [g[0], [1, c + 2.0, c + 2.0, c + 2.0], g[2]], {}
    yield "wrap", "global_id,x,y,z", [g[0], g[1], [2, L - 0.5, 5.5, 7.0]], {}
    yield "centre", "global_id,x,y,z", [[0, c, c, c + 1.0]] + g[1:], {}
    yield "fields", "global_id,x,y,z", [g[0], [1, 5.5, 6.25], g[2]], {}


@pytest.mark.parametrize("case", [v[0] for v in variants3(49)])
def test_table3_like_reference(tmp_path, case):
    L = side3("periodic", 0.007)[0]
    name, header, rows, kw = next(v for v in variants3(L) if v[0] == case)
    path = write(tmp_path / f"{name}.csv", header, rows, **kw)
    x, y, z = (np.zeros(N3, np.float32) for _ in range(3))
    h = C.c_uint64()
    rc = ref().ref_read_table3(str(path).encode(), N3, float(L), R3, fptr(x), fptr(y), fptr(z),
                               C.byref(h))
    ours = cli_hash("pfb_cell_3d", ["--N", N3, "--radius", R3, "--lambda", LAM3, "--rho", 0.007,
                                    "--t-end", 0.01, "--initial-centres", path])
    assert ours == (h.value if rc == 0 else None), case


# ---- relaxed x,y tables: substrate slab and one-layer channel ----------------------
def variants_relaxed(L):
    g = [[0, 3.5, 4.5], [1, 4.0, 4.25], [2, 30.0, 31.0]]  # no separation rule
    yield "good", "global_id,x,y", g, {}
    yield "crlf_bom", "global_id,x,y", g, {"eol": "\r\n", "bom": True}
    yield "source", "global_id,x,y", g, {"extra": [f"# source_L={L}"]}
    yield "source_bad", "global_id,x,y", g, {"extra": [f"# source_L={L + 1}"]}
    yield "source_junk", "global_id,x,y", g, {"extra": ["# source_L=4x"]}
    yield "order", "global_id,x,y", [g[0], g[2], g[1]], {}
    yield "box", "global_id,x,y", [g[0], g[1], [2, float(L), 1.0]], {}
    yield "negative", "global_id,x,y", [g[0], g[1], [2, -0.5, 1.0]], {}
    yield "long", "global_id,x,y", g + [[3, 1.0, 1.0]], {}
    yield "header", "global_id,x,y,z", g, {}


@pytest.mark.parametrize("geometry", ["slab", "channel"])
@pytest.mark.parametrize("case", [v[0] for v in variants_relaxed(50)])
def test_relaxed_tables_like_reference(tmp_path, geometry, case):
    rho = 0.05
    L, _, H, _ = side3(geometry, rho)
    name, header, rows, kw = next(v for v in variants_relaxed(L) if v[0] == case)
    path = write(tmp_path / f"{name}.csv", header, rows, **kw)
    x, y = np.zeros(N3, np.float32), np.zeros(N3, np.float32)
    ours = cli_hash("pfb_cell_3d", ["--geometry", geometry, "--N", N3, "--radius", R3, "--lambda", LAM3,
                                    "--rho", rho, "--t-end", 0.01, "--initial-centres", path])
    if geometry == "channel" and header == "global_id,x,y,z":
        return  # a channel x,y,z table: covered below
    rc = ref().ref_read_relaxed2(str(path).encode(), N3, float(L), 1 if geometry == "channel" else 0,
                                 fptr(x), fptr(y))
    if rc != 0:
        assert ours is None, case
        return
    zc = -0.5 if geometry == "slab" else 0.5 * math.ceil(2 * R3)
    assert ours == pl.table_hash(x, y, np.full(N3, zc, np.float32)), case


def variants_channel(L, H):
    c = L / 2
    g = [[0, c, c, H / 2], [1, 5.5, 6.0, 4.0], [2, 30.0, 31.0, 4.0]]
    yield "good", g
    yield "low", [g[0], [1, 5.5, 6.0, R3 - 0.25], g[2]]
    yield "floor", [g[0], [1, 5.5, 6.0, R3], g[2]]
    yield "ceiling", [g[0], [1, 5.5, 6.0, H - R3], g[2]]
    yield "high", [g[0], [1, 5.5, 6.0, H - R3 + 0.25], g[2]]
    yield "close", [g[0], [1, c + 3.0, c, H / 2], g[2]]
    yield "centre", [[0, c, c, H / 2 + 0.5]] + g[1:]


@pytest.mark.parametrize("case", [v[0] for v in variants_channel(45, 8)])
def test_channel_table_like_reference(tmp_path, case):
    rho = 0.05
    L, _, H, _ = side3("channel", rho)
    name, rows = next(v for v in variants_channel(L, H) if v[0] == case)
    path = write(tmp_path / f"{name}.csv", "global_id,x,y,z", rows)
    x, y, z = (np.zeros(N3, np.float32) for _ in range(3))
    h = C.c_uint64()
    rc = ref().ref_read_channel3(str(path).encode(), N3, float(L), H, R3, fptr(x), fptr(y), fptr(z),
                                 C.byref(h))
    ours = cli_hash("pfb_cell_3d", ["--geometry", "channel", "--N", N3, "--radius", R3, "--lambda", LAM3,
                                    "--rho", rho, "--t-end", 0.01, "--initial-centres", path])
    assert ours == (h.value if rc == 0 else None), case


def test_initial_centres_refused_on_resume(tmp_path):
    r = subprocess.run([str(LIB / "pfb_cell_3d"), "-c", str(tmp_path / "x.pf3d"), "--initial-centres",
                        str(tmp_path / "t.csv")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
    r = subprocess.run([str(LIB / "pfb_cell"), "-c", str(tmp_path / "x.bin"), "--initial-centres",
                        str(tmp_path / "t.csv")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
