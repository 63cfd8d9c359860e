"""pfb_sim2d_advance_record on a B200: the trajectory frames it writes to a
host ring without a host wait per record equal pfb_sim2d_pack_traj after
one-step advances, for intervals inside, equal to and across the six-step
graphs, into page-locked rings (written by the device, graphs included)
and pageable ones (copied), with ring wrap-around; the final state equals
a plain advance."""
import numpy as np
import pytest
import torch

import pfb200
from pfb200._abi import TRAJ_DTYPE
from helpers2d import params

pytestmark = pytest.mark.gpu


def make(p):
    cx, cy = pfb200.palmieri_centres(p.num_cells, p.L, 2.0 * p.target_radius, p.seed)
    return pfb200.Sim2D(p, cx, cy)


def pinned_ring(frames, n, pinned=True):
    if not pinned:
        return None, np.zeros((frames, n), TRAJ_DTYPE)
    t = torch.zeros((frames, n * TRAJ_DTYPE.itemsize), dtype=torch.uint8).pin_memory()
    return t, t.numpy().view(TRAJ_DTYPE).reshape(frames, n)


@pytest.fixture(scope="module")
def reference_frames():
    p = params(512, 64, seed=321)
    a = make(p)
    frames = []
    for _ in range(30):
        a.advance(1)
        frames.append(a.traj())
    state = (a.cells().tobytes(), a.phi().tobytes())
    a.close()
    return p, np.stack(frames), state


@pytest.mark.parametrize("pinned", [True, False], ids=["page-locked", "pageable"])
@pytest.mark.parametrize("every", [1, 2, 3, 4, 6, 12])
def test_frames_equal_pack_traj(reference_frames, every, pinned):
    p, ref, state = reference_frames
    b = make(p)
    n = 30 if every != 12 else 24
    keep, ring = pinned_ring(n // every, p.num_cells, pinned)
    b.advance_record(n, every, ring)
    b.sync()
    for k in range(n // every):
        assert ring[k].tobytes() == ref[(k + 1) * every - 1].tobytes(), k
    if n == 30:
        assert b.cells().tobytes() == state[0] and b.phi().tobytes() == state[1]
    assert b.step == n
    b.close()


@pytest.mark.parametrize("pinned", [True, False], ids=["page-locked", "pageable"])
def test_ring_wraps(reference_frames, pinned):
    p, ref, _ = reference_frames
    b = make(p)
    keep, ring = pinned_ring(3, p.num_cells, pinned)
    b.advance_record(7, 1, ring)   # frames 0..6 into slots k % 3
    b.sync()
    assert ring[0].tobytes() == ref[6].tobytes()
    assert ring[1].tobytes() == ref[4].tobytes()
    assert ring[2].tobytes() == ref[5].tobytes()
    # a second call continues from step 7 and counts its frames from 0
    b.advance_record(6, 2, ring)
    b.sync()
    assert ring[0].tobytes() == ref[8].tobytes()
    assert ring[1].tobytes() == ref[10].tobytes()
    assert ring[2].tobytes() == ref[12].tobytes()
    b.close()


def test_rejects_bad_arguments(reference_frames):
    p, _, _ = reference_frames
    b = make(p)
    _, ring = pinned_ring(2, p.num_cells)
    with pytest.raises(pfb200.PfbError):
        b.advance_record(4, 0, ring)
    with pytest.raises(ValueError):
        b.advance_record(4, 1, ring[0])
    assert b.step == 0
    b.close()


def test_records_start_mid_graph(reference_frames):
    """A call that starts off the six-step boundary (step 5) and records
    every 3 steps: single launches until the boundary, then record graphs."""
    p, ref, _ = reference_frames
    b = make(p)
    b.advance(5)
    keep, ring = pinned_ring(8, p.num_cells)
    b.advance_record(24, 3, ring)
    b.sync()
    for k in range(8):
        assert ring[k].tobytes() == ref[5 + 3 * (k + 1) - 1].tobytes(), k
    b.close()
