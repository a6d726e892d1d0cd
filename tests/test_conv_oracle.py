"""The corrector's CPU convolution oracle pinned by central finite differences
of its own forward pass (input and weight gradients), and its bfloat16
rounding against known values."""
import numpy as np

from oracle import conv_oracle as co


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.140625, 1e-3])
    r = co.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7 and r[3] == -2.5 and r[4] == 3.140625
    assert abs(r[5] - 1e-3) <= 1e-3 * 2 ** -8


def test_gradients_by_finite_differences():
    rng = np.random.default_rng(3)
    B, H, W, ci, cout = 2, 5, 6, 3, 4
    x = rng.normal(size=(B, H, W, ci))
    w = rng.normal(size=(cout, 9, ci))
    b = rng.normal(size=cout)
    g = rng.normal(size=(B, H, W, cout))          # dL/dy for L = sum(g * y)

    def loss(xx, ww, bb):
        return float((g * co.conv_fwd(co.pad(xx), ww, bb)).sum())

    dx = co.conv_dgrad(g, w)
    dw, db = co.conv_wgrad(co.pad(x), g)
    h = 1e-6
    for idx in [(0, 0, 0, 0), (1, 4, 5, 2), (0, 2, 3, 1)]:
        e = np.zeros_like(x)
        e[idx] = h
        fd = (loss(x + e, w, b) - loss(x - e, w, b)) / (2 * h)
        assert abs(fd - dx[idx]) <= 1e-6 * max(1.0, abs(fd))
    for idx in [(0, 0, 0), (3, 8, 2), (1, 4, 1)]:
        e = np.zeros_like(w)
        e[idx] = h
        fd = (loss(x, w + e, b) - loss(x, w - e, b)) / (2 * h)
        assert abs(fd - dw[idx]) <= 1e-6 * max(1.0, abs(fd))
    for k in range(cout):
        e = np.zeros_like(b)
        e[k] = h
        fd = (loss(x, w, b + e) - loss(x, w, b - e)) / (2 * h)
        assert abs(fd - db[k]) <= 1e-6 * max(1.0, abs(fd))


def test_gelu_grad():
    x = np.linspace(-4, 4, 33)
    h = 1e-6
    fd = (co.gelu(x + h) - co.gelu(x - h)) / (2 * h)
    assert np.max(np.abs(fd - co.gelu_grad(x))) <= 1e-8
