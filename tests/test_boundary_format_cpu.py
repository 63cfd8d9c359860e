"""PFB boundary file layout (reference common/boundary_format.h): the
72-byte header, 48-byte frame headers with the FNV-1a 64 payload checksum,
40-byte cell records, 20-byte squares and the end record; the reader
refuses corrupted payloads and files without an end record."""
import struct

import numpy as np
import pytest

from pfb200 import boundary as bf


def frame(step, cells, squares):
    payload = cells.tobytes() + b"".join(s.tobytes() for s in squares)
    head = struct.pack("<8sQdQQQ", b"PFBFRM1\0", step, step * 0.01, len(payload), len(payload),
                       bf.fnv1a64(payload))
    return head + payload


def sample(n=2, seed=0):
    rng = np.random.default_rng(seed)
    cells = np.zeros(n, bf.CELL_DTYPE)
    cells["id"] = np.arange(n)
    cells["squares"] = rng.integers(1, 5, n)
    squares = []
    for k in cells["squares"]:
        s = np.zeros(k, bf.SQUARE_DTYPE)
        s["xy"] = np.sort(rng.integers(0, 1 << 20, k)).astype(np.uint32)
        s["phi"] = rng.random((k, 4), np.float32)
        squares.append(s)
    return cells, squares


def file_bytes(frames, n=2, end=True):
    head = struct.pack("<8sIIIIIIdddQII", b"PFBND01\0", 1, 72, n, 320, 288, 20, 0.01, 1e4, 0.5,
                       7, 0, 0)
    body = b"".join(frames)
    tail = struct.pack("<8sQdQQQ", b"PFBEND1\0", 14, 0.14, 0, 0, len(frames)) if end else b""
    return head + body + tail


def test_record_sizes():
    assert bf.HEADER.size == 72 and bf.FRAME.size == 48
    assert bf.CELL_DTYPE.itemsize == 40 and bf.SQUARE_DTYPE.itemsize == 20
    assert bf.fnv1a64(b"") == 0xCBF29CE484222325
    assert bf.fnv1a64(b"a") == 0xAF63DC4C8601EC8C  # FNV-1a 64 of "a"


def test_round_trip(tmp_path):
    frames = [sample(seed=k) for k in range(3)]
    (tmp_path / "b.pfb").write_bytes(file_bytes([frame(7 * k, *f) for k, f in enumerate(frames)]))
    b = bf.read(tmp_path / "b.pfb")
    assert (b.cells, b.side, b.tile_pitch, b.level, b.interval, b.end_frames) == (2, 320, 288, 0.5, 7, 3)
    for k, (cells, squares) in enumerate(frames):
        fr = b.frames[k]
        assert fr.step == 7 * k
        np.testing.assert_array_equal(fr.cells, cells)
        for got, want in zip(fr.squares, squares):
            np.testing.assert_array_equal(got, want)


def test_refusals(tmp_path):
    good = frame(0, *sample())
    bad = bytearray(good)
    bad[-1] ^= 0xFF  # payload corrupted after the checksum was taken
    (tmp_path / "c.pfb").write_bytes(file_bytes([bytes(bad)], end=True))
    with pytest.raises(ValueError):
        bf.read(tmp_path / "c.pfb")
    (tmp_path / "e.pfb").write_bytes(file_bytes([good], end=False))
    with pytest.raises(ValueError):
        bf.read(tmp_path / "e.pfb")


def test_pfb3d_layout_and_reader(tmp_path):
    assert bf.HEADER3D.size == 128 and bf.CELL3D_DTYPE.itemsize == 64
    head = bf.HEADER3D.pack(b"PFB3D1\0\0", 1, 128, 2, 2, 3, 0, 40, 40, 56, 1.0, 1.0, 1.0, 0.01,
                            1e4, 0.5, 2, 20, 64, 0)
    cells = np.zeros(2, bf.CELL3D_DTYPE)
    cells["id"] = [0, 1]
    cells["squares"] = [1, 2]
    sq = np.zeros(3, bf.SQUARE_DTYPE)
    sq["xy"] = [5, 7, 9]
    payload = cells.tobytes() + sq.tobytes()
    frame = struct.pack("<8sQdQQQ", b"P3BFRM1\0", 4, 0.04, len(payload), len(payload),
                        bf.fnv1a64(payload)) + payload
    end = struct.pack("<8sQdQQQ", b"P3BEND1\0", 4, 0.04, 0, 0, 0)
    (tmp_path / "b").write_bytes(head + frame + end)
    b = bf.read3d(tmp_path / "b")
    assert b.complete and b.projection == 2 and b.shape == (40, 40, 56) and b.end_step == 4
    assert [list(s["xy"]) for s in b.frames[0].squares] == [[5], [7, 9]]
    (tmp_path / "u").write_bytes(head + frame)  # unterminated: an incomplete run
    assert not bf.read3d(tmp_path / "u").complete
