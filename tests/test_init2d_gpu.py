"""The 2D set-up and diagnostic passes (pfb_init_tiles2d, pfb_init_moments2d,
pfb_scatter_all2d, pfb_verify_cells2d, pfb_verify_S, pfb_pack_traj2d,
pfb_zero_u32) on a B200, through the C ABI:

* seeding and initial moments against the reference's own k_init_tiles and
  k_init_moments (oracle/_ref/libref2d.so) on the same centres: both pools
  bit-identical, origins, classes, support boxes and phi_max exact, FP64
  moments within 1e-12 relative (the sums are grouped differently);
* the aggregate rebuild exact against the integer restatement in the oracle
  and against the reference's k_scatter_all, on a state that holds every
  shape class (class 5's window starts at tile column 1);
* the invariant check, the S maximum and the trajectory records against
  numpy on the same buffers.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle2d
import pfb200
from pfb200 import CELL_DTYPE, TRAJ_DTYPE
from helpers2d import fresh_cells, params, s_from_phi, synthetic_all_classes

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not oracle2d.ref_available(), reason="reference build absent")


def seed_state(impl, p, cx, cy):
    N = p.num_cells
    dev = "cuda"
    pa = torch.full((N, 288, 288), 7.0, dtype=torch.float32, device=dev)  # junk: must be overwritten
    pb = torch.full((N, 288, 288), 7.0, dtype=torch.float32, device=dev)
    cells = torch.from_numpy(fresh_cells(p).view(np.uint8).copy()).to(dev)
    cls = torch.zeros(N, dtype=torch.uint8, device=dev)
    dcx = torch.from_numpy(np.ascontiguousarray(cx, np.float32)).to(dev)
    dcy = torch.from_numpy(np.ascontiguousarray(cy, np.float32)).to(dev)
    k = 2.7386127875258306 / p.lambda_
    reff = p.target_radius + 0.5 / k
    if impl == "pfb":
        L = pfb200.lib()
        assert L.pfb_init_tiles2d(pa.data_ptr(), pb.data_ptr(), cells.data_ptr(), cls.data_ptr(),
                                  N, p.L, dcx.data_ptr(), dcy.data_ptr(), reff, k, None) == 0
        assert L.pfb_init_moments2d(cells.data_ptr(), cls.data_ptr(), pa.data_ptr(), N, None) == 0
    else:
        R = oracle2d.rlib()
        assert R.ref2d_init_tiles(pa.data_ptr(), pb.data_ptr(), cells.data_ptr(), cls.data_ptr(),
                                  N, p.L, dcx.data_ptr(), dcy.data_ptr(), reff, k, None) == 0
        assert R.ref2d_init_moments(cells.data_ptr(), cls.data_ptr(), pa.data_ptr(), N, None) == 0
    torch.cuda.synchronize()
    return pa.cpu().numpy(), pb.cpu().numpy(), cells.cpu().numpy().view(CELL_DTYPE).copy()


@needs_ref
@pytest.mark.parametrize("L,N,seed", [(512, 64, 99), (2048, 1024, 1234), (701, 40, 5)])
def test_seed_and_moments_equal_reference_kernels(L, N, seed):
    p = params(L, N, R=12.0, seed=seed)
    cx, cy = pfb200.palmieri_centres(N, L, 24.0, seed)
    a0, a1, ca = seed_state("pfb", p, cx, cy)
    b0, b1, cb = seed_state("ref", p, cx, cy)
    assert np.array_equal(a0, b0) and np.array_equal(a1, b1)
    assert not a1.any()
    for k in ("gx0", "gy0", "cls", "cls_written", "bb_lo_x", "bb_hi_x", "bb_lo_y", "bb_hi_y",
              "promote_ctr", "phi_max", "global_id", "theta", "gamma", "v_A", "M_pf", "Ix", "Iy"):
        np.testing.assert_array_equal(ca[k], cb[k], err_msg=k)
    for k in ("V", "Cx", "Cy"):
        np.testing.assert_allclose(ca[k], cb[k], rtol=1e-12, err_msg=k)


def all_class_state(L=701):
    cells, phi = synthetic_all_classes(L=L)
    # a negative and a non-finite sample outside the windows, for the checks
    return cells, phi


def upload(cells, phi):
    c = np.ascontiguousarray(cells.copy())
    dc = torch.from_numpy(c.view(np.uint8).copy()).cuda()
    dcls = torch.from_numpy(np.ascontiguousarray(c["cls"]).astype(np.uint8)).cuda()
    dphi = torch.from_numpy(np.ascontiguousarray(phi, np.float32)).cuda()
    return dc, dcls, dphi


@pytest.mark.parametrize("L", [701, 704])
def test_scatter_all_classes_exact(L):
    cells, phi = all_class_state(L)
    P = 32 * ((L + 31) // 32)
    dc, dcls, dphi = upload(cells, phi)
    S = torch.full((L, P), 5, dtype=torch.int32, device="cuda")
    flags = torch.zeros(8, dtype=torch.int32, device="cuda")
    assert pfb200.lib().pfb_zero_u32(S.data_ptr(), L * P, None) == 0
    assert pfb200.lib().pfb_scatter_all2d(dphi.data_ptr(), dc.data_ptr(), dcls.data_ptr(),
                                          S.data_ptr(), len(cells), L, P, flags.data_ptr(),
                                          None) == 0
    got = S.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(got, s_from_phi(phi, cells, L))
    assert not flags.cpu().numpy().any()
    if oracle2d.ref_available():
        S2 = torch.zeros((L, P), dtype=torch.int32, device="cuda")
        f2 = torch.zeros(8, dtype=torch.int32, device="cuda")
        assert oracle2d.rlib().ref2d_scatter_all(dphi.data_ptr(), dc.data_ptr(), dcls.data_ptr(),
                                                 S2.data_ptr(), len(cells), L, P, f2.data_ptr(),
                                                 None) == 0
        np.testing.assert_array_equal(got, S2.cpu().numpy().view(np.uint32))


def test_scatter_raises_overflow_and_clamp():
    cells, phi = all_class_state(701)
    L, P = 701, 704
    phi = phi.copy()
    wx, wy, tx0, ty0 = pfb200.CLASSES[int(cells["cls"][2])]
    phi[2, ty0 + 5, tx0 + 7] = 3.0  # 3^2 > 4: clamped
    dc, dcls, dphi = upload(cells, phi)
    S = torch.zeros((L, P), dtype=torch.int32, device="cuda")
    gy, gx = (cells["gy0"][2] + 5) % L, (cells["gx0"][2] + 7) % L
    S[gy, gx] = -1  # 0xFFFFFFFF: the next add wraps
    flags = torch.zeros(8, dtype=torch.int32, device="cuda")
    assert pfb200.lib().pfb_scatter_all2d(dphi.data_ptr(), dc.data_ptr(), dcls.data_ptr(),
                                          S.data_ptr(), len(cells), L, P, flags.data_ptr(),
                                          None) == 0
    f = flags.cpu().numpy()
    assert f[pfb200.FLAG_NAMES.index("S_overflow")] == 1
    assert f[pfb200.FLAG_NAMES.index("q_clamp")] == 1


def test_verify_and_max_and_traj():
    cells, phi = all_class_state(701)
    phi = phi.copy()
    phi[1, 3, 5] = -0.25            # outside every window (rows 0..31 are outside all classes but 5)
    phi[4, 10, 280] = float("nan")  # outside: passed over, as the reference's fmaxf fold does
    dc, dcls, dphi = upload(cells, phi)
    N = len(cells)
    V = torch.zeros(N, dtype=torch.float64, device="cuda")
    O = torch.zeros(N, dtype=torch.float32, device="cuda")
    assert pfb200.lib().pfb_verify_cells2d(dphi.data_ptr(), dc.data_ptr(), dcls.data_ptr(), N,
                                           V.data_ptr(), O.data_ptr(), None) == 0
    eV, eO = np.zeros(N), np.zeros(N, np.float32)
    for n in range(N):
        wx, wy, tx0, ty0 = pfb200.CLASSES[int(cells["cls"][n])]
        t = phi[n].astype(np.float64)
        inside = np.zeros((288, 288), bool)
        inside[ty0:ty0 + wy, tx0:tx0 + wx] = True
        eV[n] = (t[inside] ** 2).sum()
        out = np.abs(t[~inside])
        eO[n] = np.nanmax(out) if out.size else 0.0
    np.testing.assert_allclose(V.cpu().numpy(), eV, rtol=1e-13)
    np.testing.assert_array_equal(O.cpu().numpy(), eO)
    assert eO[1] == np.float32(0.25)
    # S maximum over an odd word count and an unaligned start
    S = torch.randint(0, 2**31 - 1, (100003,), dtype=torch.int64).to(torch.int32).cuda()
    for off, n in ((0, 100003), (1, 99999), (0, 3)):
        m = torch.zeros(1, dtype=torch.int32, device="cuda")
        assert pfb200.lib().pfb_verify_S(S.data_ptr() + 4 * off, n, m.data_ptr(), None) == 0
        want = S.cpu().numpy().view(np.uint32)[off:off + n].max()
        assert int(m.cpu().numpy().view(np.uint32)[0]) == int(want)
    # trajectory records
    L = 701
    c = cells.copy()
    c["vx"], c["vy"], c["perim"] = 0.25, -0.5, 3.5
    dc, dcls, _ = upload(c, phi)
    out = torch.zeros(N * TRAJ_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    assert pfb200.lib().pfb_pack_traj2d(dc.data_ptr(), dcls.data_ptr(), out.data_ptr(), N, L,
                                        None) == 0
    t = out.cpu().numpy().view(TRAJ_DTYPE)
    px = c["gx0"] + c["Cx"] / c["V"]
    py = c["gy0"] + c["Cy"] / c["V"]
    np.testing.assert_array_equal(t["cx"], (px - np.floor(px / L) * L).astype(np.float32))
    np.testing.assert_array_equal(t["cy"], (py - np.floor(py / L) * L).astype(np.float32))
    np.testing.assert_array_equal(t["global_id"], c["global_id"])
    np.testing.assert_array_equal(t["cls"], c["cls"])
    for k_out, k_in in (("vx", "vx"), ("vy", "vy"), ("theta", "theta"), ("gamma", "gamma"),
                        ("v_A", "v_A"), ("phi_max", "phi_max")):
        np.testing.assert_array_equal(t[k_out], c[k_in], err_msg=k_out)
    np.testing.assert_array_equal(t["volume"], c["V"].astype(np.float32))
    np.testing.assert_array_equal(t["perim"], c["perim"].astype(np.float32))
    st = (C.c_uint * 1)()
    assert pfb200.lib().pfb_device_status(st, 0) == 0 and st[0] == 0
