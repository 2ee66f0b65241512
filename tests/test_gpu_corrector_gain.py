"""What the trained corrector gains over the method without it.

A network trained with this library's BF16 kernels on coarse (64^2) / fine
(256^2) pairs of the seeded Euler four-quadrant family predicts the one-step
residual (block-averaged fine state minus plain coarse step) of seeds it never
saw: its relative L2 error is clearly below 1, the error of the plain step
(no correction).  Rollout accuracy and time are measured by
classic_b200.learn on the full-size family, not here."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_corrector_beats_the_plain_step_on_unseen_pairs():
    from classic_b200 import corrector as C
    from classic_b200 import learn as L

    rng = np.random.default_rng(0)
    n = 64
    x, t, _ = L.generate(list(range(10000, 10016)), C.default_norm(), n, 12, rng)
    assert x.shape[0] >= 100
    norm = L.recalibrate(x, t, C.default_norm())
    t.clamp_(-5.0, 5.0)
    C.project_tiles(t)
    net = C.ConvNet(seed=0)
    losses = C.train(net, x, t, iters=1500, batch=16, crop=32, lr=1e-3, noise=0.01, delta=1.0,
                     log=lambda it, l: None)
    assert losses[-1][1] < losses[0][1]

    # pairs of unseen seeds, in the training scaling
    xv, tv, _ = L.generate(list(range(40000, 40004)), C.Norm(C.default_norm().values), n, 6, rng)
    sc = C.default_norm().values
    for c in range(8):
        xv[..., c] = (xv[..., c].float() * float(norm.values[4 + c] / sc[4 + c])).to(xv.dtype)
    for c in range(4):
        tv[..., c] *= float(norm.values[12 + c] / sc[12 + c])
    tv.clamp_(-5.0, 5.0)
    C.project_tiles(tv)
    err = C.one_step_gain(net, xv, tv)
    print(f"one-step relative error on unseen pairs: {err:.3f} (plain step: 1)")
    assert err < 0.85
