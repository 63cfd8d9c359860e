"""Batched ensemble: systems of different sizes advanced by one launch per
step evolve exactly (bit for bit) as each system run alone, and the
replicas-one-at-a-time path gives the same state."""
import numpy as np
import pytest

import pfb200
from helpers2d import params

pytestmark = pytest.mark.gpu

SYSTEMS = [(300, 8, 11), (384, 16, 12), (512, 30, 13), (512, 64, 14), (768, 40, 15)]


def make(seed_shift=0, storage=0):
    ps, cs = [], []
    for L, N, seed in SYSTEMS:
        p = params(L, N, seed=seed + seed_shift, phi_storage=storage)
        ps.append(p)
        cs.append(pfb200.palmieri_centres(N, L, p.target_radius, p.seed))
    return ps, cs


def state(sim):
    return sim.cells().tobytes(), sim.phi().tobytes(), sim.S().tobytes(), sim.flags().tobytes()


@pytest.mark.parametrize("storage", [0, 1, 2])
def test_batched_systems_match_systems_run_alone(storage):
    """Binary32, binary16 and bfloat16 pools (the 16-bit ensembles round
    with the same hash of seed, step, cell and pixel as a system alone)."""
    ps, cs = make(storage=storage)
    ens = pfb200.Ensemble2D(ps, cs)
    ens.advance(37)
    assert ens.step == 37
    for r, (p, c) in enumerate(zip(ps, cs)):
        alone = pfb200.Sim2D(p, c[0], c[1])
        alone.advance(37)
        got = state(ens.system(r))
        want = state(alone)
        for g, w, name in zip(got, want, ("cells", "phi", "S", "flags")):
            assert g == w, f"system {r}: {name} differs"
        alone.close()
    ens.close()


@pytest.mark.parametrize("cluster", [2, 4])
def test_serial_and_batched_paths_agree(cluster):
    ps, cs = make(100)
    a = pfb200.Ensemble2D(ps, cs, cluster=cluster)
    b = pfb200.Ensemble2D(ps, cs, cluster=cluster)
    a.advance(13)
    b.advance_serial(13)
    for r in range(len(ps)):
        assert state(a.system(r)) == state(b.system(r)), r
    a.close()
    b.close()


@pytest.mark.parametrize("storage", [0, 2])
def test_autotune_picks_a_cluster_size(storage):
    ps, cs = make(200, storage)
    e = pfb200.Ensemble2D(ps, cs)
    k = e.autotune(6)
    assert k in ((2, 4, 8) if storage == 0 else (2, 4))
    assert all(int(e.system(r).flags().sum()) == 0 for r in range(len(ps)))
    e.close()


@pytest.mark.parametrize("pinned", [True, False], ids=["page-locked", "pageable"])
@pytest.mark.parametrize("every", [1, 3, 4])
def test_advance_record_frames(every, pinned):
    """pfb_ens2d_advance_record: frame k holds every system's trajectory
    records (system 0 first) after step (k + 1) * every, as each system's
    pfb_sim2d_pack_traj after one-step advances gives them."""
    import torch
    from pfb200._abi import TRAJ_DTYPE
    ps, cs = make(seed_shift=3)
    a = pfb200.Ensemble2D(ps, cs)
    b = pfb200.Ensemble2D(ps, cs)
    n = 24
    want = []
    for _ in range(n):
        a.advance(1)
        a.sync()
        want.append(np.concatenate([a.system(r).traj() for r in range(len(ps))]))
    frames = n // every
    if pinned:
        buf = torch.zeros((frames, b.total_cells * TRAJ_DTYPE.itemsize), dtype=torch.uint8).pin_memory()
        ring = buf.numpy().view(TRAJ_DTYPE).reshape(frames, b.total_cells)
    else:
        ring = np.zeros((frames, b.total_cells), TRAJ_DTYPE)
    b.advance_record(n, every, ring)
    b.sync()
    assert b.step == n
    for k in range(frames):
        assert ring[k].tobytes() == want[(k + 1) * every - 1].tobytes(), k
    for r in range(len(ps)):
        assert state(a.system(r)) == state(b.system(r))
    a.close()
    b.close()
