"""FP64 CPU oracle of the surrogate U-Net (test infrastructure only: the
network's tensor-core forward and backward passes are checked against it;
nothing in the product calls it).

Same architecture and flat parameter layout as the library's pfb_sur2d:
eight 3x3 "same" convolutions (per layer: weights [cout][cin][3][3] then the
bias), ReLU after all but the last, a 2x2 average pool after the second and a
nearest upsampling plus skip connection before the fifth. The loss is the
mean over images and pixels of (out[..., 0] - target)^2. Built on
conv_oracle; pinned by finite differences in the CPU tests.
"""
from __future__ import annotations

import numpy as np

import conv_oracle as co

# (cin, cout, relu) per layer, padded channel counts
LAYERS = [(16, 32, True), (32, 32, True), (32, 32, True), (32, 32, True),
          (32, 32, True), (32, 32, True), (32, 32, True), (32, 16, False)]


def num_params() -> int:
    return sum(9 * ci * co_ + co_ for ci, co_, _ in LAYERS)


def unpack(flat: np.ndarray) -> list[tuple[np.ndarray, np.ndarray]]:
    out, off = [], 0
    for ci, cout, _ in LAYERS:
        w = flat[off:off + 9 * ci * cout].reshape(cout, ci, 3, 3)
        off += 9 * ci * cout
        b = flat[off:off + cout]
        off += cout
        out.append((w, b))
    return out


def pack(layers: list[tuple[np.ndarray, np.ndarray]]) -> np.ndarray:
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in layers])


def _pool(a):
    B, H, W, C = a.shape
    return a.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def _up(a):
    return a.repeat(2, axis=1).repeat(2, axis=2)


def _sum2(a):
    B, H, W, C = a.shape
    return a.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def forward(flat: np.ndarray, x: np.ndarray):
    """x (B, H, W, 16) -> out (B, H, W, 16) and the activations."""
    L = unpack(np.asarray(flat, np.float64))
    relu = lambda v: np.maximum(v, 0.0)  # noqa: E731
    a1 = relu(co.conv3x3(x, *L[0]))
    a2 = relu(co.conv3x3(a1, *L[1]))
    p = _pool(a2)
    a3 = relu(co.conv3x3(p, *L[2]))
    a4 = relu(co.conv3x3(a3, *L[3]))
    u = _up(a4) + a2
    a5 = relu(co.conv3x3(u, *L[4]))
    a6 = relu(co.conv3x3(a5, *L[5]))
    a7 = relu(co.conv3x3(a6, *L[6]))
    out = co.conv3x3(a7, *L[7])
    return out, dict(x=np.asarray(x, np.float64), a1=a1, a2=a2, p=p, a3=a3, a4=a4, u=u, a5=a5,
                     a6=a6, a7=a7)


def loss(out: np.ndarray, target: np.ndarray) -> float:
    return float(np.mean((out[..., 0] - target) ** 2))


def loss_and_grad(flat: np.ndarray, x: np.ndarray, target: np.ndarray):
    """(loss, flat gradient) of the mean-squared error."""
    L = unpack(np.asarray(flat, np.float64))
    out, c = forward(flat, x)
    go = np.zeros_like(out)
    go[..., 0] = 2.0 * (out[..., 0] - target) / target.size
    g = [None] * 8
    g[7] = co.conv3x3_wgrad(c["a7"], go)
    d = co.conv3x3_dgrad(go, L[7][0]) * (c["a7"] > 0)
    g[6] = co.conv3x3_wgrad(c["a6"], d)
    d = co.conv3x3_dgrad(d, L[6][0]) * (c["a6"] > 0)
    g[5] = co.conv3x3_wgrad(c["a5"], d)
    d = co.conv3x3_dgrad(d, L[5][0]) * (c["a5"] > 0)
    g[4] = co.conv3x3_wgrad(c["u"], d)
    gu = co.conv3x3_dgrad(d, L[4][0])
    d = _sum2(gu) * (c["a4"] > 0)
    g[3] = co.conv3x3_wgrad(c["a3"], d)
    d = co.conv3x3_dgrad(d, L[3][0]) * (c["a3"] > 0)
    g[2] = co.conv3x3_wgrad(c["p"], d)
    gp = co.conv3x3_dgrad(d, L[2][0])
    d = (0.25 * _up(gp) + gu) * (c["a2"] > 0)
    g[1] = co.conv3x3_wgrad(c["a1"], d)
    d = co.conv3x3_dgrad(d, L[1][0]) * (c["a1"] > 0)
    g[0] = co.conv3x3_wgrad(c["x"], d)
    return loss(out, target), pack(g)
