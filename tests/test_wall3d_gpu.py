"""Channel wall diagnostics (reference k_measure_wall_diagnostics,
src/pf3d/kernels.cu): per cell, the sum over its in-domain voxels of phi^2
times the binary32 wall profile psi_w^2(z), and of phi^2 outside the slit,
against a numpy FP64 restatement on the same field (FP64 sums in a
different grouping: relative 1e-12)."""
import math

import numpy as np
import pytest

import pfb200

from helpers3d import small_centres, small_params

pytestmark = pytest.mark.gpu


def wall_psi_sq(p):
    k = math.sqrt(7.5) / p.wall_width
    lo, hi = float(p.channel_padding), float(p.channel_padding + p.channel_height)
    out = np.zeros(p.Nz, np.float32)
    for z in range(p.Nz):
        c = z + 0.5
        fluid = 0.25 * (1.0 + math.tanh(k * (c - lo))) * (1.0 - math.tanh(k * (c - hi)))
        out[z] = np.float32((1.0 - fluid) ** 2)
    return out


def test_wall_diagnostics_match_numpy():
    p = small_params("channel")
    sim = pfb200.Sim3D(p, small_centres(p))
    sim.advance(4)
    sim.measure_wall()
    cells, phi = sim.cells(), sim.phi()
    psi = wall_psi_sq(p).astype(np.float64)
    B = sim.B
    for i in range(p.num_cells):
        z = int(cells["origin_z"][i]) + np.arange(B)
        inside = (z >= 0) & (z < p.Nz)
        sq = phi[i].astype(np.float64) ** 2  # [z, y, x]
        per_plane = sq.sum(axis=(1, 2))
        overlap = float((per_plane[inside] * psi[z[inside]]).sum())
        slit = (z >= p.channel_padding) & (z < p.channel_padding + p.channel_height)
        outside = float(per_plane[inside & ~slit].sum())
        np.testing.assert_allclose(cells["wall_overlap"][i], overlap, rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(cells["outside_slit_volume"][i], outside, rtol=1e-12, atol=1e-300)
    assert cells["wall_overlap"].max() > 0.0
    sim.close()


def test_wall_diagnostics_need_a_channel():
    p = small_params("periodic")
    sim = pfb200.Sim3D(p, small_centres(p))
    with pytest.raises(RuntimeError):
        sim.measure_wall()
    sim.close()
