"""PFVMOM4 file layout (reference common/velocity_format.h): the 56-byte
header with its field offsets, frames of an int64 step and cells x 26
float64 columns; the reader refuses other files and partial frames."""
import struct

import numpy as np
import pytest

from pfb200 import velocity as vf


def write(path, cells, frames, tail=b""):
    head = struct.pack("<8sIIdqdIIQ", b"PFVMOM4\0", cells, 26, 0.01, 40, 320.0, 3, 2, 4)
    body = b"".join(struct.pack("<q", s) + rows.astype("<f8").tobytes() for s, rows in frames)
    path.write_bytes(head + body + tail)


def test_header_layout():
    assert vf.HEADER.size == 56
    raw = vf.HEADER.pack(b"PFVMOM4\0", 1, 26, 0.5, 7, 9.0, 3, 2, 11)
    assert raw[:8] == b"PFVMOM4\0"
    assert struct.unpack_from("<I", raw, 8)[0] == 1       # cells
    assert struct.unpack_from("<d", raw, 16)[0] == 0.5    # dt
    assert struct.unpack_from("<q", raw, 24)[0] == 7      # start step
    assert struct.unpack_from("<d", raw, 32)[0] == 9.0    # side
    assert struct.unpack_from("<I", raw, 40)[0] == 3      # spatial stride
    assert struct.unpack_from("<Q", raw, 48)[0] == 11     # dense start


def test_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    frames = [(40 + 5 * k, rng.normal(size=(3, 26))) for k in range(4)]
    write(tmp_path / "v.bin", 3, frames)
    f = vf.read(tmp_path / "v.bin")
    assert (f.cells, f.dt, f.start_step, f.side, f.spatial_stride, f.quadrature, f.dense_start) == \
        (3, 0.01, 40, 320.0, 3, 2, 4)
    np.testing.assert_array_equal(f.steps, [40, 45, 50, 55])
    for k, (_, rows) in enumerate(frames):
        np.testing.assert_array_equal(f.rows[k], rows)


def test_refuses_partial_frames_and_other_files(tmp_path):
    write(tmp_path / "v.bin", 2, [(0, np.zeros((2, 26)))], tail=b"\0" * 9)
    with pytest.raises(ValueError):
        vf.read(tmp_path / "v.bin")
    (tmp_path / "w.bin").write_bytes(b"PFVMOM3\0" + b"\0" * 48)
    with pytest.raises(ValueError):
        vf.read(tmp_path / "w.bin")
