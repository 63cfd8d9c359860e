"""tcgen05 convolutions (forward, data gradient, weight gradient) against the
FP64 oracle on the same bfloat16 inputs and weights.

The kernels read bfloat16 operands and accumulate in binary32; the oracle
gets the same bfloat16-rounded values in float64, so the only difference is
the binary32 accumulation. Tolerance: 1e-5 of the sum of absolute terms
(the oracle run on |x| and |w|) plus 1e-6."""
import ctypes as C

import numpy as np
import pytest

import conv_oracle as co
import pfb200
from pfb200 import check, lib

pytestmark = pytest.mark.gpu

PAIRS = [(16, 32), (32, 32), (32, 16), (16, 16)]
SHAPES = [(3, 64, 64), (4, 32, 32), (2, 9, 13)]


def torch():
    import torch as t
    return t


def bf16_round(a: np.ndarray) -> np.ndarray:
    t = torch()
    return t.from_numpy(np.ascontiguousarray(a, np.float32)).to(t.bfloat16).float().numpy()


def dev_bf16(a: np.ndarray):
    t = torch()
    return t.from_numpy(np.ascontiguousarray(a, np.float32)).to(t.bfloat16).cuda().contiguous()


def dev_f32(a: np.ndarray):
    t = torch()
    return t.from_numpy(np.ascontiguousarray(a, np.float32)).cuda().contiguous()


def pack(w: np.ndarray, transpose: bool):
    t = torch()
    cout, cin = w.shape[:2]
    wd = dev_f32(w)
    p = t.zeros(9 * cin * cout, dtype=t.bfloat16, device="cuda")
    check(lib().pfb_conv3x3_pack(wd.data_ptr(), p.data_ptr(), cin, cout, int(transpose), None), "pack")
    return p, wd


def status_ok():
    v = C.c_uint()
    check(lib().pfb_conv_status(C.byref(v), 1), "status")
    return v.value == 0


def inputs(B, H, W, cin, cout, seed):
    rng = np.random.default_rng(seed)
    x = bf16_round(rng.standard_normal((B, H, W, cin)))
    w = (rng.standard_normal((cout, cin, 3, 3)) / np.sqrt(9 * cin)).astype(np.float32)
    b = rng.standard_normal(cout).astype(np.float32)
    return x, w, b


@pytest.mark.parametrize("cin,cout", PAIRS)
@pytest.mark.parametrize("B,H,W", SHAPES)
def test_forward_vs_fp64(cin, cout, B, H, W):
    t = torch()
    x, w, b = inputs(B, H, W, cin, cout, 11 + cin + cout + H)
    wq = bf16_round(w)
    xd = dev_bf16(co.to_padded(x))
    p, _ = pack(w, False)
    bd = dev_f32(b)
    P2 = (H + 2) * (W + 2)
    yf = t.full((B, P2, cout), 7.0, dtype=t.float32, device="cuda")
    y = t.zeros((B, P2, cout), dtype=t.bfloat16, device="cuda")
    check(lib().pfb_conv3x3_forward(xd.data_ptr(), y.data_ptr(), yf.data_ptr(), p.data_ptr(),
                                    bd.data_ptr(), None, B, H, W, cin, cout, 0, None), "forward")
    t.cuda.synchronize()
    assert status_ok()
    got = co.from_padded(yf.cpu().numpy(), H, W)
    ref = co.conv3x3(x, wq, b)
    scale = co.conv3x3(np.abs(x), np.abs(wq)) + np.abs(b)
    err = np.abs(got - ref)
    assert np.all(err <= 1e-5 * scale + 1e-6), float((err / (scale + 1e-30)).max())
    g = yf.cpu().numpy().reshape(B, H + 2, W + 2, cout)
    assert not g[:, 1:H + 1, 0].any() and not g[:, 1:H + 1, W + 1].any()  # border columns zeroed
    assert np.all(g[:, 0] == 7.0) and np.all(g[:, H + 1] == 7.0)          # border rows untouched
    yb = co.from_padded(y.float().cpu().numpy(), H, W)
    np.testing.assert_array_equal(yb, bf16_round(got))


@pytest.mark.parametrize("cin,cout", [(32, 32), (16, 32)])
def test_forward_relu_and_gate(cin, cout):
    t = torch()
    B, H, W = 2, 32, 32
    x, w, b = inputs(B, H, W, cin, cout, 5)
    wq = bf16_round(w)
    rng = np.random.default_rng(9)
    gate = bf16_round(rng.standard_normal((B, H, W, cout)))
    xd, gd = dev_bf16(co.to_padded(x)), dev_bf16(co.to_padded(gate))
    p, _ = pack(w, False)
    bd = dev_f32(b)
    yf = t.zeros((B, (H + 2) * (W + 2), cout), dtype=t.float32, device="cuda")
    check(lib().pfb_conv3x3_forward(xd.data_ptr(), None, yf.data_ptr(), p.data_ptr(), bd.data_ptr(),
                                    gd.data_ptr(), B, H, W, cin, cout, 1, None), "forward")
    t.cuda.synchronize()
    got = co.from_padded(yf.cpu().numpy(), H, W)
    ref = np.maximum(co.conv3x3(x, wq, b), 0.0) * (gate > 0)
    scale = co.conv3x3(np.abs(x), np.abs(wq)) + np.abs(b)
    assert np.all(np.abs(got - ref) <= 1e-5 * scale + 1e-6)


@pytest.mark.parametrize("cin,cout", PAIRS)
@pytest.mark.parametrize("B,H,W", SHAPES[:2])
def test_data_gradient_vs_fp64(cin, cout, B, H, W):
    """dX = forward(dY, flipped transposed W): cout -> cin channels."""
    t = torch()
    _, w, _ = inputs(B, H, W, cin, cout, 21 + H)
    wq = bf16_round(w)
    rng = np.random.default_rng(4 + cin)
    dy = bf16_round(rng.standard_normal((B, H, W, cout)))
    p, _ = pack(w, True)
    dyd = dev_bf16(co.to_padded(dy))
    dx = t.zeros((B, (H + 2) * (W + 2), cin), dtype=t.float32, device="cuda")
    check(lib().pfb_conv3x3_forward(dyd.data_ptr(), None, dx.data_ptr(), p.data_ptr(), None, None,
                                    B, H, W, cout, cin, 0, None), "dgrad")
    t.cuda.synchronize()
    assert status_ok()
    got = co.from_padded(dx.cpu().numpy(), H, W)
    ref = co.conv3x3_dgrad(dy, wq)
    scale = co.conv3x3_dgrad(np.abs(dy), np.abs(wq))
    assert np.all(np.abs(got - ref) <= 1e-5 * scale + 1e-6)


@pytest.mark.parametrize("cx,cy", PAIRS)
@pytest.mark.parametrize("B,H,W", SHAPES)
def test_weight_gradient_vs_fp64(cx, cy, B, H, W):
    t = torch()
    rng = np.random.default_rng(31 + cx + cy + W)
    x = bf16_round(rng.standard_normal((B, H, W, cx)))
    dy = bf16_round(rng.standard_normal((B, H, W, cy)))
    xd, dyd = dev_bf16(co.to_padded(x)), dev_bf16(co.to_padded(dy))
    nbytes = lib().pfb_conv3x3_wgrad_workspace(B, H, W, cx, cy)
    ws = t.zeros(nbytes // 4, dtype=t.float32, device="cuda")
    dw = t.zeros((cy, cx, 3, 3), dtype=t.float32, device="cuda")
    db = t.zeros(cy, dtype=t.float32, device="cuda")
    for _ in range(2):  # twice in a row: the result is overwritten, not accumulated
        check(lib().pfb_conv3x3_wgrad(xd.data_ptr(), dyd.data_ptr(), ws.data_ptr(), nbytes,
                                      dw.data_ptr(), db.data_ptr(), B, H, W, cx, cy, None), "wgrad")
    t.cuda.synchronize()
    assert status_ok()
    rdw, rdb = co.conv3x3_wgrad(x, dy)
    sdw, sdb = co.conv3x3_wgrad(np.abs(x), np.abs(dy))
    assert np.all(np.abs(dw.cpu().numpy() - rdw) <= 1e-5 * sdw + 1e-5)
    assert np.all(np.abs(db.cpu().numpy() - rdb) <= 1e-5 * sdb + 1e-5)


def test_weight_gradient_is_deterministic():
    t = torch()
    B, H, W, cx, cy = 6, 64, 64, 32, 32
    rng = np.random.default_rng(2)
    xd = dev_bf16(co.to_padded(rng.standard_normal((B, H, W, cx))))
    dyd = dev_bf16(co.to_padded(rng.standard_normal((B, H, W, cy))))
    nbytes = lib().pfb_conv3x3_wgrad_workspace(B, H, W, cx, cy)
    ws = t.zeros(nbytes // 4, dtype=t.float32, device="cuda")
    outs = []
    for _ in range(3):
        dw = t.zeros((cy, cx, 3, 3), dtype=t.float32, device="cuda")
        check(lib().pfb_conv3x3_wgrad(xd.data_ptr(), dyd.data_ptr(), ws.data_ptr(), nbytes,
                                      dw.data_ptr(), None, B, H, W, cx, cy, None), "wgrad")
        outs.append(dw.cpu().numpy().tobytes())
    assert outs[0] == outs[1] == outs[2]


def test_rejects_unbuilt_channels_and_small_workspace():
    with pytest.raises(pfb200.PfbError):
        check(lib().pfb_conv3x3_forward(8, 16, None, 32, None, None, 1, 8, 8, 8, 32, 0, None), "f")
    with pytest.raises(pfb200.PfbError):
        check(lib().pfb_conv3x3_wgrad(16, 16, 16, 4, 16, None, 1, 8, 8, 32, 32, None), "w")


@pytest.mark.parametrize("cin,cout,B,H,W", [(32, 32, 600, 32, 32), (16, 32, 40, 64, 64),
                                            (32, 16, 7, 30, 124), (32, 32, 3, 20, 126)])
def test_pipelined_forward_equals_one_tile_per_cta(cin, cout, B, H, W):
    """The persistent warp-specialised forward (TMA ring, two TMEM
    accumulators; W <= 124) and the one-tile-per-CTA kernel give the same
    bits, including when each CTA walks many tiles (600 images) and at the
    widths on either side of the TMA box limit."""
    t = torch()
    x, w, b = inputs(B, H, W, cin, cout, 5 + cin + W)
    xd = dev_bf16(co.to_padded(x))
    p, _ = pack(w, False)
    bd = dev_f32(b)
    P2 = (H + 2) * (W + 2)
    outs = []
    try:
        for pipe in (2, 0):
            check(lib().pfb_conv_set_pipeline(pipe), "pipeline")
            yf = t.full((B, P2, cout), 7.0, dtype=t.float32, device="cuda")
            y = t.zeros((B, P2, cout), dtype=t.bfloat16, device="cuda")
            check(lib().pfb_conv3x3_forward(xd.data_ptr(), y.data_ptr(), yf.data_ptr(), p.data_ptr(),
                                            bd.data_ptr(), None, B, H, W, cin, cout, 1, None), "forward")
            t.cuda.synchronize()
            assert status_ok()
            outs.append((yf.cpu().numpy(), y.float().cpu().numpy()))
    finally:
        check(lib().pfb_conv_set_pipeline(1), "pipeline")
    assert outs[0][0].tobytes() == outs[1][0].tobytes()
    assert outs[0][1].tobytes() == outs[1][1].tobytes()
