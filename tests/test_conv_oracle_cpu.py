"""The FP64 convolution oracle (oracle/conv_oracle.py) against central finite
differences of its own forward pass: pins the data and weight gradients the
tensor-core kernels are checked against."""
import numpy as np

import conv_oracle as co


def _setup(seed=3, B=2, H=5, W=7, cin=3, cout=4):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((B, H, W, cin))
    w = rng.standard_normal((cout, cin, 3, 3))
    b = rng.standard_normal(cout)
    dy = rng.standard_normal((B, H, W, cout))
    return x, w, b, dy


def test_forward_matches_direct_sum():
    x, w, b, _ = _setup()
    y = co.conv3x3(x, w, b)
    B, H, W, cin = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    i, j, o = 2, 0, 3
    ref = b[o] + sum(xp[1, i + ky, j + kx, c] * w[o, c, ky, kx]
                     for c in range(cin) for ky in range(3) for kx in range(3))
    assert abs(y[1, i, j, o] - ref) < 1e-12


def test_data_gradient_by_finite_differences():
    x, w, b, dy = _setup()
    dx = co.conv3x3_dgrad(dy, w)
    h = 1e-6
    for idx in [(0, 0, 0, 0), (1, 4, 6, 2), (0, 2, 3, 1)]:
        xp, xm = x.copy(), x.copy()
        xp[idx] += h
        xm[idx] -= h
        fd = ((co.conv3x3(xp, w, b) - co.conv3x3(xm, w, b)) * dy).sum() / (2 * h)
        assert abs(fd - dx[idx]) < 1e-6 * max(1.0, abs(fd))


def test_weight_gradient_by_finite_differences():
    x, w, b, dy = _setup()
    dw, db = co.conv3x3_wgrad(x, dy)
    h = 1e-6
    for idx in [(0, 0, 0, 0), (3, 2, 2, 1), (1, 1, 1, 2)]:
        wp, wm = w.copy(), w.copy()
        wp[idx] += h
        wm[idx] -= h
        fd = ((co.conv3x3(x, wp, b) - co.conv3x3(x, wm, b)) * dy).sum() / (2 * h)
        assert abs(fd - dw[idx]) < 1e-6 * max(1.0, abs(fd))
    bp = b.copy()
    bp[2] += h
    bm = b.copy()
    bm[2] -= h
    fd = ((co.conv3x3(x, w, bp) - co.conv3x3(x, w, bm)) * dy).sum() / (2 * h)
    assert abs(fd - db[2]) < 1e-6 * max(1.0, abs(fd))


def test_padded_layout_round_trip():
    x, _, _, _ = _setup()
    p = co.to_padded(x)
    assert p.shape == (2, 7 * 9, 3)
    np.testing.assert_array_equal(co.from_padded(p, 5, 7), x)
    q = p.reshape(2, 7, 9, 3)
    assert not q[:, 0].any() and not q[:, -1].any() and not q[:, :, 0].any() and not q[:, :, -1].any()
