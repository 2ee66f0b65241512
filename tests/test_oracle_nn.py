"""The corrector network's NumPy oracle checked on its own: its backward
pass equals finite differences of its forward pass (float64, no BF16
rounding), and the flipped-weight convolution is the adjoint."""
import numpy as np

import nn_oracle as O


def _net(rng, cin=3, hid=4, cout=2):
    return [(rng.standard_normal((hid, 9, cin)) * 0.3, rng.standard_normal(hid) * 0.1, 1),
            (rng.standard_normal((hid, 9, hid)) * 0.3, rng.standard_normal(hid) * 0.1, 1),
            (rng.standard_normal((cout, 9, hid)) * 0.3, rng.standard_normal(cout) * 0.1, 0)]


def _forward64(x, layers):
    a = x
    cache = []
    for w, b, act in layers:
        z = O.conv3x3(a, w, b)
        cache.append((a, z))
        a = O.gelu(z) if act else z
    return a, cache


def _backward64(dy, layers, cache):
    grads = [None] * len(layers)
    d = dy
    for k in range(len(layers) - 1, -1, -1):
        w, b, act = layers[k]
        a_in, z = cache[k]
        dz = d * O.gelu_grad(z) if act else d
        grads[k] = O.conv3x3_wgrad(a_in, dz)
        d = O.conv3x3(dz, O.flip(w))
    return grads


def test_backward_equals_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((1, 5, 6, 3))
    target = rng.standard_normal((1, 5, 6, 2))
    layers = _net(rng)

    def loss(ls):
        y, _ = _forward64(x, ls)
        return float(((y - target) ** 2).sum())

    y, cache = _forward64(x, layers)
    grads = _backward64(2.0 * (y - target), layers, cache)
    eps = 1e-6
    for k, (w, b, act) in enumerate(layers):
        for idx in [(0, 4, 0), (1, 0, 1), (w.shape[0] - 1, 8, w.shape[2] - 1)]:
            wp = w.copy(); wp[idx] += eps
            wm = w.copy(); wm[idx] -= eps
            lp = loss([(wp, b, act) if j == k else l for j, l in enumerate(layers)])
            lm = loss([(wm, b, act) if j == k else l for j, l in enumerate(layers)])
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - grads[k][0][idx]) <= 1e-6 * max(1.0, abs(fd))
        bp = b.copy(); bp[0] += eps
        bm = b.copy(); bm[0] -= eps
        fd = (loss([(w, bp, act) if j == k else l for j, l in enumerate(layers)]) -
              loss([(w, bm, act) if j == k else l for j, l in enumerate(layers)])) / (2 * eps)
        assert abs(fd - grads[k][1][0]) <= 1e-6 * max(1.0, abs(fd))


def test_flip_is_adjoint():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 7, 5, 3))
    dz = rng.standard_normal((2, 7, 5, 4))
    w = rng.standard_normal((4, 9, 3))
    lhs = np.sum(O.conv3x3(x, w) * dz)
    rhs = np.sum(x * O.conv3x3(dz, O.flip(w)))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0], dtype=np.float32)
    r = O.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and r[3] == -2.5 and r[4] == 0.0
