"""The FP64 U-Net oracle (oracle/unet_oracle.py) against central finite
differences of its own loss, on 8 x 8 images: pins the network gradients the
tensor-core training step is checked against."""
import numpy as np

import unet_oracle as uo


def _setup(seed=5):
    rng = np.random.default_rng(seed)
    flat = rng.standard_normal(uo.num_params()) * 0.2
    x = np.zeros((2, 8, 8, 16))
    x[..., :2] = rng.random((2, 8, 8, 2))
    t = rng.standard_normal((2, 8, 8)) * 0.1
    return flat, x, t


def test_parameter_count_and_layout():
    assert uo.num_params() == sum(9 * a * b + b for a, b, _ in uo.LAYERS)
    flat = np.arange(uo.num_params(), dtype=np.float64)
    np.testing.assert_array_equal(uo.pack(uo.unpack(flat)), flat)


def test_gradient_by_finite_differences():
    flat, x, t = _setup()
    _, g = uo.loss_and_grad(flat, x, t)
    rng = np.random.default_rng(1)
    offs = np.cumsum([0] + [9 * a * b + b for a, b, _ in uo.LAYERS])
    h = 1e-5
    for l in range(8):
        # one weight on a used input channel and the first bias of each layer
        for i in (offs[l] + rng.integers(0, 9 * 2), offs[l + 1] - uo.LAYERS[l][1]):
            fp, fm = flat.copy(), flat.copy()
            fp[i] += h
            fm[i] -= h
            out_p, _ = uo.forward(fp, x)
            out_m, _ = uo.forward(fm, x)
            fd = (uo.loss(out_p, t) - uo.loss(out_m, t)) / (2 * h)
            assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (l, i, fd, g[i])
