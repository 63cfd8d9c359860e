"""PFB boundary files (reference common/boundary_format.h): a 72-byte
little-endian header, independently framed snapshots, and an end record;
and their 3D form PFB3D (common/boundary_format_3d.h, `read3d`).

A frame's payload is `cells` 40-byte cell records (id, tile origin x/y,
periodic centroid x/y, gamma, mobility, active speed, target radius, square
count) followed by the squares of each cell in record order: 20 bytes each,
the tile position packed as x | y << 16 and the four binary32 corners (lower
left, lower right, upper right, upper left) of a 2x2 square that phi = 1/2
crosses. The frame header carries the FNV-1a 64 checksum of the payload.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HEADER = struct.Struct("<8sIIIIIIdddQII")
FRAME = struct.Struct("<8sQdQQQ")
assert HEADER.size == 72 and FRAME.size == 48

CELL_DTYPE = np.dtype([("id", "<i4"), ("origin_x", "<i4"), ("origin_y", "<i4"), ("cx", "<f4"),
                       ("cy", "<f4"), ("gamma", "<f4"), ("mobility", "<f4"),
                       ("active_speed", "<f4"), ("radius", "<f4"), ("squares", "<u4")])
SQUARE_DTYPE = np.dtype([("xy", "<u4"), ("phi", "<f4", 4)])
assert CELL_DTYPE.itemsize == 40 and SQUARE_DTYPE.itemsize == 20


def fnv1a64(data: bytes) -> int:
    h = 14695981039346656037
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


@dataclass
class Frame:
    step: int
    time: float
    checksum: int
    cells: np.ndarray                      # CELL_DTYPE records
    squares: list = field(default_factory=list)  # per cell, SQUARE_DTYPE arrays
    payload: bytes = b""


@dataclass
class BoundaryFile:
    cells: int
    side: int
    tile_pitch: int
    dt: float
    tau: float
    level: float
    interval: int
    codec: int
    frames: list
    end_step: int
    end_time: float
    end_frames: int


def read(path, verify: bool = True) -> BoundaryFile:
    data = Path(path).read_bytes()
    (magic, version, hbytes, cells, side, pitch, sq_bytes, dt, tau, level, interval, codec,
     _) = HEADER.unpack_from(data, 0)
    if magic != b"PFBND01\0" or version != 1 or hbytes != 72 or sq_bytes != 20:
        raise ValueError("not a PFB file")
    if codec != 0:
        raise ValueError("compressed PFB frames are not supported by this reader")
    pos, frames = 72, []
    while True:
        if pos + FRAME.size > len(data):
            raise ValueError("PFB file has no end record")
        tag, step, time, raw, stored, checksum = FRAME.unpack_from(data, pos)
        pos += FRAME.size
        if tag == b"PFBEND1\0":
            if pos != len(data):
                raise ValueError("bytes after the PFB end record")
            return BoundaryFile(cells, side, pitch, dt, tau, level, interval, codec, frames,
                                step, time, checksum)
        if tag != b"PFBFRM1\0" or raw != stored or pos + raw > len(data):
            raise ValueError("malformed PFB frame")
        payload = data[pos:pos + raw]
        pos += raw
        if verify and fnv1a64(payload) != checksum:
            raise ValueError(f"PFB frame at step {step}: checksum mismatch")
        meta = np.frombuffer(payload, CELL_DTYPE, count=cells)
        sq = np.frombuffer(payload, SQUARE_DTYPE, offset=cells * 40)
        if int(meta["squares"].astype(np.int64).sum()) != sq.size:
            raise ValueError("PFB frame square count mismatch")
        edges = np.concatenate([[0], np.cumsum(meta["squares"].astype(np.int64))])
        frames.append(Frame(step, time, checksum, meta.copy(),
                            [sq[edges[i]:edges[i + 1]].copy() for i in range(cells)], payload))


# ---- PFB3D ------------------------------------------------------------------
HEADER3D = struct.Struct("<8sIIIIIIqqqddddddQIIQ")
assert HEADER3D.size == 128
CELL3D_DTYPE = np.dtype([("id", "<i8"), ("origin_x", "<i8"), ("origin_y", "<i8"),
                         ("origin_z", "<i8"), ("brick_edge", "<u4"), ("plane_edge", "<u4"),
                         ("squares", "<u4"), ("reserved", "<u4"), ("gamma", "<f4"),
                         ("active_speed", "<f4"), ("radius", "<f4"), ("reserved_float", "<f4")])
assert CELL3D_DTYPE.itemsize == 64


@dataclass
class BoundaryFile3D:
    cells: int
    projection: int      # 1 basal, 2 maximum
    boundary_flags: int
    shape: tuple         # (nx, ny, nz)
    dt: float
    tau: float
    level: float
    interval: int
    codec: int
    frames: list
    complete: bool       # an end record closes the file
    end_step: int = -1
    end_time: float = 0.0


def read3d(path, verify: bool = True) -> BoundaryFile3D:
    data = Path(path).read_bytes()
    (magic, version, hbytes, cells, proj, flags, codec, nx, ny, nz, dx, dy, dz, dt, tau, level,
     interval, sq_bytes, cell_bytes, _) = HEADER3D.unpack_from(data, 0)
    if magic != b"PFB3D1\0\0" or version != 1 or hbytes != 128 or sq_bytes != 20 or cell_bytes != 64:
        raise ValueError("not a PFB3D file")
    if codec != 0:
        raise ValueError("compressed PFB3D frames are not supported by this reader")
    out = BoundaryFile3D(cells, proj, flags, (nx, ny, nz), dt, tau, level, interval, codec, [], False)
    pos = 128
    while pos < len(data):
        if pos + FRAME.size > len(data):
            raise ValueError("truncated PFB3D frame header")
        tag, step, time, raw, stored, checksum = FRAME.unpack_from(data, pos)
        pos += FRAME.size
        if tag == b"P3BEND1\0":
            if pos != len(data):
                raise ValueError("bytes after the PFB3D end record")
            out.complete, out.end_step, out.end_time = True, step, time
            return out
        if tag != b"P3BFRM1\0" or raw != stored or pos + raw > len(data):
            raise ValueError("malformed PFB3D frame")
        payload = data[pos:pos + raw]
        pos += raw
        if verify and fnv1a64(payload) != checksum:
            raise ValueError(f"PFB3D frame at step {step}: checksum mismatch")
        meta = np.frombuffer(payload, CELL3D_DTYPE, count=cells)
        sq = np.frombuffer(payload, SQUARE_DTYPE, offset=cells * 64)
        if int(meta["squares"].astype(np.int64).sum()) != sq.size:
            raise ValueError("PFB3D frame square count mismatch")
        edges = np.concatenate([[0], np.cumsum(meta["squares"].astype(np.int64))])
        out.frames.append(Frame(step, time, checksum, meta.copy(),
                                [sq[edges[i]:edges[i + 1]].copy() for i in range(cells)], payload))
    return out
