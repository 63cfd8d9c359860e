"""PFVMOM4 velocity-component files (reference common/velocity_format.h): a
56-byte little-endian header, then frames of an int64 step and cells x 26
float64 columns.

Columns: 0 cell id, 1-2 periodic centroid, 3 polarity angle, 4 gamma,
5 phase-field mobility, 6 active speed, 7 volume, 8 observed steps, 9-20 the
integral channels (active, interaction, interfacial, overlap, area,
advection correction; x/y pairs), 21 spatial samples, 22-25 the current
interfacial and overlap rates.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np

COLUMNS = 26
HEADER = struct.Struct("<8sIIdqdIIQ")
assert HEADER.size == 56


@dataclass
class VelocityFile:
    cells: int
    dt: float
    start_step: int
    side: float
    spatial_stride: int
    quadrature: int
    dense_start: int
    steps: np.ndarray   # (frames,) int64
    rows: np.ndarray    # (frames, cells, 26) float64


def read(path) -> VelocityFile:
    data = Path(path).read_bytes()
    if len(data) < HEADER.size:
        raise ValueError("not a PFVMOM4 file")
    magic, cells, columns, dt, start, side, stride, quad, dense = HEADER.unpack_from(data, 0)
    if magic != b"PFVMOM4\0" or columns != COLUMNS:
        raise ValueError("not a PFVMOM4 file")
    frame = 8 + cells * COLUMNS * 8
    body = data[HEADER.size:]
    if len(body) % frame:
        raise ValueError("partial PFVMOM4 frame")
    n = len(body) // frame
    raw = np.frombuffer(body, np.uint8).reshape(n, frame)
    steps = raw[:, :8].copy().view("<i8").reshape(n)
    rows = raw[:, 8:].copy().view("<f8").reshape(n, cells, COLUMNS)
    return VelocityFile(cells, dt, start, side, stride, quad, dense, steps, rows)
