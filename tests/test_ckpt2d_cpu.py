"""The reference's 2D checkpoint file (PF "CELL" schema 1) on the CPU:
layout, write -> read -> write byte identity, and the reference's acceptance
rules (reference src/checkpoint.cu:348-615 reader, 823-1011 writer). States
come from the CPU oracle's fresh start."""
import struct

import numpy as np
import pytest

import oracle2d
import pfb200
from helpers2d import fresh_cells, params
from pfb200 import checkpoint as ck

N = 3


@pytest.fixture(scope="module")
def state():
    p = params(320, N, R=12.0, seed=21)
    cx, cy = pfb200.palmieri_centres(N, p.L, 24.0, p.seed)
    cells, phi = oracle2d.init_state(p.to_c(), cx, cy, fresh_cells(p))
    cells["vx"] = np.linspace(-0.01, 0.01, N)
    cells["perim"] = 75.0
    return p, cells, phi


def write(tmp_path, state, step=0, name="a.bin"):
    p, cells, phi = state
    rec = ck.params_record(p)
    path = tmp_path / name
    ck.write(path, rec, step, cells, phi)
    return path, rec


def test_layout(tmp_path, state):
    p, cells, phi = state
    path, rec = write(tmp_path, state, step=0)
    b = path.read_bytes()
    tile = 288 * 288 * 4
    assert len(b) == 44 + 192 + 4 + 12 + N * (96 + tile) + 5 * (8 + 4 * N)
    magic, schema, step, t, n, save, zero, traj = struct.unpack_from("<IIidiiii", b, 0)
    assert (magic, schema, step, n, save, zero, traj) == (0x43454C4C, 1, 0, N, 0, 0, 100)
    assert b[36:40] == b"\0\0\0\0" and struct.unpack_from("<I", b, 40)[0] == 192
    r = b[44:236]
    assert struct.unpack_from("<ii", r, 0) == (p.L, p.L)
    assert struct.unpack_from("<d", r, 88)[0] == p.target_radius
    assert struct.unpack_from("<Q", r, 136)[0] == p.seed
    assert struct.unpack_from("<i", b, 236)[0] == 288
    assert struct.unpack_from("<iii", b, 240) == (1, 0, N)
    h = b[252:252 + 96]
    cid, ox, oy, cls = struct.unpack_from("<iiii", h, 0)
    assert cid == 0 and cls == int(cells["cls"][0])
    assert ox == (int(cells["gx0"][0]) - 64) % p.L
    assert struct.unpack_from("<d", h, 40)[0] == cells["V"][0]
    assert struct.unpack_from("<f", h, 88)[0] == cells["phi_max"][0]
    off = 252 + N * (96 + tile)
    magics = [struct.unpack_from("<Ii", b, off + k * (8 + 4 * N)) for k in range(5)]
    assert [m for m, _ in magics] == [0x504F4C52, 0x47414D41, 0x56415F41, 0x52414449, 0x4D4F4249]
    assert all(c == N for _, c in magics)


def test_round_trip_is_byte_identical(tmp_path, state):
    p, cells, phi = state
    path, rec = write(tmp_path, state, step=4)
    got = ck.read(path)
    assert got.step == 4 and got.time == 4 * p.dt and got.had_mobility
    np.testing.assert_array_equal(got.phi, phi)
    for f in ("gx0", "gy0", "cls", "V", "Cx", "Cy", "perim", "bb_lo_x", "bb_hi_x", "bb_lo_y",
              "bb_hi_y", "vx", "vy", "phi_max", "gamma", "v_A", "R_tgt", "theta", "M_pf",
              "global_id", "promote_ctr"):
        np.testing.assert_array_equal(got.cells[f], cells[f], err_msg=f)
    assert not got.cells["tumble_ctr"].any() and not got.cells["Ix"].any()
    again = tmp_path / "b.bin"
    ck.write(again, got.params, got.step, got.cells, got.phi)
    assert again.read_bytes() == path.read_bytes()
    assert not (tmp_path / "b.bin.tmp").exists()


def _mutated(tmp_path, src, fn, name="m.bin"):
    b = bytearray(src.read_bytes())
    b = fn(b)
    q = tmp_path / name
    q.write_bytes(bytes(b))
    return q


def _rejects(path, match):
    with pytest.raises(pfb200.PfbError, match=match):
        ck.read(path)


def _put(fmt, off, val):
    def f(b):
        struct.pack_into(fmt, b, off, val)
        return b
    return f


def test_rejections(tmp_path, state):
    path, _ = write(tmp_path, state, step=2)
    tile = 288 * 288 * 4
    cell0 = 252
    side = cell0 + N * (96 + tile)
    blk = 8 + 4 * N
    cases = [
        (_put("<I", 0, 0x12345678), "not a cell checkpoint"),
        (_put("<I", 4, 2), "schema"),
        (_put("<i", 28, 1), "fixed checkpoint metadata"),
        (_put("<i", 24, 1), "internally inconsistent"),
        (_put("<B", 37, 1), "fixed checkpoint metadata"),
        (_put("<I", 40, 191), "parameter record"),
        (_put("<i", 44 + 180, 3), "internally inconsistent"),
        (_put("<i", 236, 256), "tile pitch"),
        (_put("<i", 240, 2), "single-GPU"),
        (_put("<d", 12, 0.5), "step \\* dt"),
        (_put("<d", 44 + 8, 2.0), "dx and dy"),
        (_put("<i", cell0, 5), "ids must be"),
        (_put("<i", cell0 + 20, 1), "invalid state metadata"),
        (_put("<f", cell0 + 24, 3.0), "centroid"),
        (_put("<f", cell0 + 88, 0.5), "disagrees"),
        (_put("<i", cell0 + 72, 0), "disagrees"),
        (_put("<f", cell0 + 96 + 4 * (288 * 10 + 10), float("nan")), "not finite"),
        (lambda b: b[:cell0 + 96 + 100], "short read"),
        (lambda b: b[:side + 3 * blk], "missing required sidecars: RADI"),
        (lambda b: b + b[side:side + blk], "duplicate"),
        (_put("<I", side, 0x41424344), "unsupported sidecar"),
        (_put("<i", side + 4, N + 1), "entries"),
        (_put("<f", side + 2 * blk + 8, -1.0), "invalid value"),
        (_put("<f", side + blk + 8, 0.0), "invalid value"),
        (_put("<f", side + blk + 8, 1000.0), "laplacian bound"),
    ]
    for k, (fn, match) in enumerate(cases):
        _rejects(_mutated(tmp_path, path, fn, f"m{k}.bin"), match)


def test_missing_mobility_defaults_to_half(tmp_path, state):
    path, _ = write(tmp_path, state)
    tile = 288 * 288 * 4
    side = 252 + N * (96 + tile)
    q = _mutated(tmp_path, path, lambda b: b[:side + 4 * (8 + 4 * N)], "nomobi.bin")
    got = ck.read(q)
    assert not got.had_mobility
    assert np.all(got.cells["M_pf"] == np.float32(0.5))
    # sidecars in another order are accepted
    b = path.read_bytes()
    blocks = [b[side + k * (8 + 4 * N): side + (k + 1) * (8 + 4 * N)] for k in range(5)]
    r = tmp_path / "reordered.bin"
    r.write_bytes(b[:side] + b"".join(reversed(blocks)))
    np.testing.assert_array_equal(ck.read(r).cells["theta"], ck.read(path).cells["theta"])


def test_writer_refusals(tmp_path, state):
    p, cells, phi = state
    rec = ck.params_record(p)
    bad = cells.copy()
    bad["global_id"][1] = 7
    with pytest.raises(pfb200.PfbError, match="carries id"):
        ck.write(tmp_path / "x.bin", rec, 0, bad, phi)
    bad = cells.copy()
    bad["cls_written"][0, 1] = 2
    with pytest.raises(pfb200.PfbError, match="written class"):
        ck.write(tmp_path / "x.bin", rec, 1, bad, phi)
    with pytest.raises(pfb200.PfbError, match="int32"):
        ck.write(tmp_path / "x.bin", rec, 2 ** 31, cells, phi)
    assert not (tmp_path / "x.bin").exists() and not (tmp_path / "x.bin.tmp").exists()


def test_reference_written_file_reads_and_rewrites_byte_identically(tmp_path):
    """tests/golden/ckpt2d_ref_n2.bin.gz was written by the reference's
    cell_gh200 (tests/golden/make_ckpt2d_fixture.sh): 2 cells, 301^2, step 3."""
    import gzip
    from pathlib import Path
    raw = gzip.decompress((Path(__file__).parent / "golden" / "ckpt2d_ref_n2.bin.gz").read_bytes())
    src = tmp_path / "ref.bin"
    src.write_bytes(raw)
    got = ck.read(src)
    assert got.step == 3 and got.cells.size == 2 and got.had_mobility
    assert got.params.Nx == 301 and got.params.target_radius == 12.0 and got.params.seed == 3
    assert np.all(got.cells["V"] > 400.0) and np.all(got.cells["M_pf"] == np.float32(0.5))
    out = tmp_path / "again.bin"
    ck.write(out, got.params, got.step, got.cells, got.phi)
    assert out.read_bytes() == raw
