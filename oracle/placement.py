"""ORACLE -- test infrastructure only (tests/ import it; nothing in the product
does). A plain-Python restatement of the reference's fresh-start placements
for checking the command-line programs' initial state:

* ``MT19937_64``: the 64-bit Mersenne Twister with the parameters and seeding
  the C++ standard fixes for ``std::mt19937_64`` (pinned by the standard's
  known answer: the 10000th output for the default seed 5489 is
  9981545732273789042);
* ``palmieri2d``: sequential periodic placement in a square
  (reference include/palmieri_initializer.hpp:48-96), used by the slab;
* ``palmieri3d``: the periodic cube (include/pf3d/palmieri_initializer.hpp:
  56-125);
* ``channel3d``: the hard-wall slit (include/pf3d/palmieri_initializer.hpp:
  349-410);
* ``table_hash``: FNV-1a 64 over int64 id and binary32 x, y, z rows
  (include/pf3d/initializer.hpp:97-124).

Pure-Python loops: for the small populations of the tests.
"""
from __future__ import annotations

import math
import struct

import numpy as np

_M64 = (1 << 64) - 1


class MT19937_64:
    """std::mt19937_64: w=64, n=312, m=156, r=31, a=0xB5026F5AA96619E9,
    u=29 d=0x5555555555555555, s=17 b=0x71D67FFFEDA60000, t=37
    c=0xFFF7EEE000000000, l=43, f=6364136223846793005."""

    N, M = 312, 156
    UPPER, LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF

    def __init__(self, seed: int = 5489):
        mt = [seed & _M64]
        for i in range(1, self.N):
            prev = mt[-1]
            mt.append((6364136223846793005 * (prev ^ (prev >> 62)) + i) & _M64)
        self.mt, self.i = mt, self.N

    def _twist(self):
        mt = self.mt
        for k in range(self.N):
            y = (mt[k] & self.UPPER) | (mt[(k + 1) % self.N] & self.LOWER)
            v = mt[(k + self.M) % self.N] ^ (y >> 1)
            mt[k] = v ^ 0xB5026F5AA96619E9 if y & 1 else v
        self.i = 0

    def __call__(self) -> int:
        if self.i >= self.N:
            self._twist()
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & _M64


def u53(g: MT19937_64) -> float:
    return float(g() >> 11) * 2.0 ** -53


def f32(v: float) -> float:
    return float(np.float32(v))


def min_image(d: float, side: float) -> float:
    return d - side * math.floor(d / side + 0.5)


def palmieri2d(n: int, side: float, radius: float, seed: int):
    x, y = [f32(0.5 * side)], [f32(0.5 * side)]
    g = MT19937_64(seed)
    while len(x) < n:
        cx, cy = side * u53(g), side * u53(g)
        if all(not (min_image(cx - x[j], side) ** 2 + min_image(cy - y[j], side) ** 2 < radius * radius)
               for j in range(len(x))):
            x.append(f32(cx))
            y.append(f32(cy))
    return np.array(x, np.float32), np.array(y, np.float32)


def palmieri3d(n: int, side: float, radius: float, seed: int):
    x, y, z = [f32(0.5 * side)], [f32(0.5 * side)], [f32(0.5 * side)]
    g = MT19937_64(seed)
    r2 = radius * radius
    while len(x) < n:
        cx, cy, cz = side * u53(g), side * u53(g), side * u53(g)
        ok = True
        for j in range(len(x)):
            dx, dy, dz = (min_image(cx - x[j], side), min_image(cy - y[j], side),
                          min_image(cz - z[j], side))
            if dx * dx + dy * dy + dz * dz < r2:
                ok = False
                break
        if ok:
            x.append(f32(cx))
            y.append(f32(cy))
            z.append(f32(cz))
    return tuple(np.array(v, np.float32) for v in (x, y, z))


def channel3d(n: int, side: float, height: int, radius: float, seed: int):
    """Centres in slit coordinates (z measured from the lower wall)."""
    lo, hi = radius, float(height) - radius
    x, y, z = [f32(0.5 * side)], [f32(0.5 * side)], [f32(0.5 * height)]
    g = MT19937_64(seed)
    r2 = radius * radius
    while len(x) < n:
        cx, cy = f32(side * u53(g)), f32(side * u53(g))
        cz = f32(lo + (hi - lo) * u53(g))
        ok = True
        for j in range(len(x)):
            dx, dy, dz = min_image(cx - x[j], side), min_image(cy - y[j], side), cz - z[j]
            if dx * dx + dy * dy + dz * dz < r2:
                ok = False
                break
        if ok:
            x.append(cx)
            y.append(cy)
            z.append(cz)
    return tuple(np.array(v, np.float32) for v in (x, y, z))


def table_hash(x, y, z) -> int:
    h = 0xCBF29CE484222325
    for i in range(len(x)):
        row = struct.pack("<qfff", i, float(x[i]), float(y[i]), float(z[i]))
        for b in row:
            h = ((h ^ b) * 0x100000001B3) & _M64
    return h


def domain3d(geometry: str, n: int, radius: float, rho: float, lam: float,
             height: int = 0, slab_height: int = 0, auto_brick: int = 0):
    """Lateral side and Nz of a fresh run (reference include/pf3d/params.cuh:
    224-268, src/pf3d/main.cu:712-832). Channel: height defaults to
    ceil(2R); returns (side, Nz, H, padding) with padding ceil(3 lambda)."""
    sphere = 4.0 * math.pi * radius * radius * radius / 3.0
    if geometry == "slab":
        side = math.ceil(math.sqrt(n * (math.pi * radius * radius) / rho))
        return side, slab_height or 2 * auto_brick, 0, 0
    if geometry == "channel":
        H = height or int(math.ceil(2.0 * radius))
        pad = int(math.ceil(3.0 * lam))
        side = math.ceil(math.sqrt(n * sphere / (rho * H)))
        return side, H + 2 * pad, H, pad
    side = math.ceil(math.cbrt(n * sphere / rho))
    return side, side, 0, 0
