"""The reference's 3D checkpoint file (PF3D schema 1) on the CPU: the
CRC-64/ECMA-182 against its published check value, layout, write -> read ->
write byte identity, and the reference's acceptance rules (reference
src/pf3d/checkpoint.cu:116-420, 599-1235). States are synthetic spheres on
base bricks (the reader checks records and sizes, not the physics)."""
import ctypes as C
import math
import struct

import numpy as np
import pytest

import pfb200
from pfb200 import checkpoint as ck
from pfb200 import CELL3D_DTYPE

B = 64


def make_state(geometry="periodic", n=2):
    p = pfb200.SimParams3D(Nx=96, Ny=96, Nz=96 if geometry == "periodic" else 128,
                           geometry=geometry, num_cells=n, target_radius=10.0, seed=4)
    k = math.sqrt(7.5) / p.lambda_
    z, y, x = np.meshgrid(np.arange(B), np.arange(B), np.arange(B), indexing="ij")
    phi = np.zeros((n, B, B, B), np.float32)
    cells = np.zeros(n, CELL3D_DTYPE)
    for i in range(n):
        c = (31.6 + i * 0.3, 32.2, 31.9)
        r = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
        phi[i] = 0.5 * (1.0 - np.tanh(k * (r - 10.4)))
        w = phi[i].astype(np.float64)
        cells[i]["global_id"] = i
        cells[i]["origin_x"], cells[i]["origin_y"] = 10 + 40 * i, -7
        cells[i]["origin_z"] = 3 if geometry == "periodic" else 2
        th = 0.4 + i
        if geometry == "slab":
            cells[i]["polarity_x"], cells[i]["polarity_y"] = math.cos(th), math.sin(th)
        else:
            cells[i]["polarity_x"], cells[i]["polarity_y"], cells[i]["polarity_z"] = 0.6, 0.0, 0.8
        cells[i]["velocity_x"] = 1e-3 * (i + 1)
        cells[i]["gamma"], cells[i]["v_A"], cells[i]["R_tgt"] = 1.0, 0.01, 10.0
        cells[i]["phi_max"] = float(phi[i].max())
        cells[i]["V"] = (w * w).sum()
        cells[i]["Cx"] = (w * w * x).sum()
        cells[i]["surface"] = 1234.5
        cells[i]["Ix"] = 1e-4 * i
        cells[i]["tumble_ctr"] = 3 * i
        sup = np.argwhere(w > 1e-5)
        (lz, ly, lx), (hz, hy, hx) = sup.min(0), sup.max(0)
        cells[i]["bb_lo_x"], cells[i]["bb_hi_x"] = lx, hx
        cells[i]["bb_lo_y"], cells[i]["bb_hi_y"] = ly, hy
        cells[i]["bb_lo_z"], cells[i]["bb_hi_z"] = lz, hz
        cells[i]["pending_shift_x"] = 1
    return p, cells, phi


def test_crc64_ecma_check_value():
    data = b"123456789"
    assert pfb200.lib().pfb_crc64_ecma(0, data, len(data)) == 0x6C40DF5F0B497347
    assert pfb200.lib().pfb_crc64_ecma(0, b"", 0) == 0
    # incremental update equals one pass
    a = pfb200.lib().pfb_crc64_ecma(0, data[:4], 4)
    assert pfb200.lib().pfb_crc64_ecma(a, data[4:], 5) == 0x6C40DF5F0B497347


@pytest.mark.parametrize("geometry", ["periodic", "slab"])
def test_layout_and_round_trip(tmp_path, geometry):
    p, cells, phi = make_state(geometry)
    rec = ck.params_record3d(p, B)
    path = tmp_path / "c.pf3d"
    ck.write3d(path, rec, 7, cells, phi, 4)
    b = path.read_bytes()
    n = cells.size
    assert len(b) == 96 + 288 + n * (256 + 4 * B ** 3)
    magic, ver, hb, endian, dims, scalar, flags = struct.unpack_from("<IHHIIII", b, 0)
    assert (magic, ver, hb, endian, dims, scalar, flags) == (0x44334650, 1, 96, 0x01020304, 3, 1, 3)
    step, t, cn = struct.unpack_from("<qdQ", b, 24)
    assert (step, cn) == (7, n) and t == 7 * p.dt
    assert struct.unpack_from("<IIII", b, 48) == (288, 256, B, 1)
    assert struct.unpack_from("<QQ", b, 64) == (B ** 3, 4 * B ** 3)
    crc, shards = struct.unpack_from("<QQ", b, 80)
    assert shards == 4
    zeroed = b[:80] + b"\0" * 8 + b[88:]
    assert pfb200.lib().pfb_crc64_ecma(0, zeroed, len(zeroed)) == crc
    got = ck.read3d(path)
    assert got.step == 7 and got.brick_edge == B and got.base_measure_shards == 4
    np.testing.assert_array_equal(got.phi, phi)
    for f in ("global_id", "origin_x", "origin_y", "origin_z", "polarity_x", "polarity_z", "velocity_x",
              "gamma", "v_A", "R_tgt", "phi_max", "V", "Cx", "surface", "Ix", "tumble_ctr", "bb_lo_x",
              "bb_hi_z", "pending_shift_x"):
        np.testing.assert_array_equal(got.cells[f], cells[f], err_msg=f)
    again = tmp_path / "d.pf3d"
    ck.write3d(again, got.params, got.step, got.cells, got.phi, got.base_measure_shards)
    assert again.read_bytes() == b


def _rejects(tmp_path, src, fn, match, name):
    b = bytearray(src.read_bytes())
    b = fn(b)
    q = tmp_path / name
    q.write_bytes(bytes(b))
    with pytest.raises(pfb200.PfbError, match=match):
        ck.read3d(q)


def _put(fmt, off, val):
    def f(b):
        struct.pack_into(fmt, b, off, val)
        return b
    return f


def test_rejections(tmp_path):
    p, cells, phi = make_state()
    path = tmp_path / "c.pf3d"
    ck.write3d(path, ck.params_record3d(p, B), 2, cells, phi, 4)
    c0 = 96 + 288
    cases = [
        (_put("<I", 0, 0x4C4C4543), "not a PF3D"),
        (_put("<H", 4, 2), "schema"),
        (_put("<I", 48, 287), "record-size"),
        (_put("<I", 20, 1), "checksum flag"),
        (_put("<Q", 88, 65), "shard count"),
        (_put("<d", 32, 0.5), "step \\* dt"),
        (_put("<I", 96 + 208, 2), "integrator"),
        (_put("<d", 96 + 24, 2.0), "dx, dy and dz"),
        (_put("<q", c0, 5), "carries id"),
        (_put("<f", c0 + 32, 0.9), "invalid"),
        (_put("<I", c0 + 144, 1 << 3), "invalid"),
        (_put("<I", c0 + 188, 1), "reserved"),
        (_put("<Q", c0 + 200, 1), "reserved"),
        (_put("<i", c0 + 172, B + 1), "invalid"),
        (_put("<i", c0 + 152, B), "invalid"),
        # a 72^3 payload would run into the next record
        (_put("<I", c0 + 184, 72), "carries id|storage edge|truncates"),
        (_put("<I", c0 + 184, 100), "storage edge"),
        (_put("<f", c0 + 256 + 4 * 1000, 0.123), "CRC"),
        (lambda b: b[:-4], "bytes"),
        (lambda b: b + b"\0\0\0\0", "bytes"),
    ]
    for k, (fn, match) in enumerate(cases):
        _rejects(tmp_path, path, fn, match, f"m{k}.pf3d")


def promote_cell(cells, phi, n, edge):
    """Cell n moved into a centred cube of `edge` padded with exact zeros, its
    world field unchanged (the reference's adaptive resize)."""
    off = (edge - B) // 2
    cube = np.zeros((edge, edge, edge), np.float32)
    cube[off:off + B, off:off + B, off:off + B] = phi[n]
    c = cells.copy()
    for k in "xyz":
        c["origin_" + k][n] -= off
        c["C" + k][n] += off * c["V"][n]
        c["bb_lo_" + k][n] += off
        c["bb_hi_" + k][n] += off
    c["storage_edge"][n] = edge
    return c, cube


def test_promoted_cube_round_trip(tmp_path):
    """A cell on a promoted cube (storage_edge 80 > B = 64): its record stores
    the cube's edge and is followed by 80^3 values (reference
    src/pf3d/checkpoint.cu:655-751); the file reads back and re-writes byte for
    byte, and a base record reads with storage_edge 0."""
    p, cells, phi = make_state()
    c, cube = promote_cell(cells, phi, 1, 80)
    packed = np.concatenate([phi[0].ravel(), cube.ravel()])
    path = tmp_path / "p.pf3d"
    ck.write3d(path, ck.params_record3d(p, B), 5, c, packed, 4)
    b = path.read_bytes()
    assert len(b) == 96 + 288 + 2 * 256 + 4 * (B ** 3 + 80 ** 3)
    assert struct.unpack_from("<I", b, 96 + 288 + 184)[0] == B
    assert struct.unpack_from("<I", b, 96 + 288 + 256 + 4 * B ** 3 + 184)[0] == 80
    got = ck.read3d(path)
    assert list(got.cells["storage_edge"]) == [0, 80]
    assert list(got.edges()) == [B, 80]
    f = got.fields()
    np.testing.assert_array_equal(f[0], phi[0])
    np.testing.assert_array_equal(f[1], cube)
    with pytest.raises(ValueError):
        got.phi
    again = tmp_path / "q.pf3d"
    ck.write3d(again, got.params, got.step, got.cells, got.packed, got.base_measure_shards)
    assert again.read_bytes() == b


def test_writer_refusals(tmp_path):
    p, cells, phi = make_state()
    rec = ck.params_record3d(p, B)
    bad = cells.copy()
    bad["flags"][0] = 1  # a fatal flag
    with pytest.raises(pfb200.PfbError, match="refused"):
        ck.write3d(tmp_path / "x.pf3d", rec, 0, bad, phi, 4)
    with pytest.raises(pfb200.PfbError, match="shards"):
        ck.write3d(tmp_path / "x.pf3d", rec, 0, cells, phi, 0)
    assert not (tmp_path / "x.pf3d").exists()


def test_reference_written_file_reads_and_rewrites_byte_identically(tmp_path):
    """tests/golden/ckpt3d_ref_n2.pf3d.gz was written by the reference's
    cell_gh200_3d (tests/golden/make_ckpt3d_fixture.sh): 2 periodic cells of
    radius 4 in 32^3 bricks on 48^3, step 3; its CRC is the reference's."""
    import gzip
    from pathlib import Path
    raw = gzip.decompress((Path(__file__).parent / "golden" / "ckpt3d_ref_n2.pf3d.gz").read_bytes())
    src = tmp_path / "ref.pf3d"
    src.write_bytes(raw)
    got = ck.read3d(src)
    assert got.step == 3 and got.cells.size == 2 and got.brick_edge == 32
    assert got.params.Nx == got.params.Ny == got.params.Nz == 48
    assert got.params.boundary_flags == 0x7 and got.params.target_radius == 4.0
    assert np.all(got.cells["V"] > 200.0)
    out = tmp_path / "again.pf3d"
    ck.write3d(out, got.params, got.step, got.cells, got.phi, got.base_measure_shards)
    assert out.read_bytes() == raw
