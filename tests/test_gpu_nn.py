"""The corrector's device kernels (include/claw_nn.h) against the NumPy oracle
(oracle/nn_oracle.py): forward convolutions, weight and data gradients, the
whole network's backward pass, and the solver glue.  BF16 storage is
emulated in the oracle at the same places, so the remaining differences are
FP32 accumulation order and the last BF16 rounding."""
import ctypes

import numpy as np
import pytest

import nn_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _lib():
    from classic_b200 import _lib
    return _lib.load()


def _p(t):
    """Device pointer of a tensor; the caller keeps the tensor alive (a
    temporary's memory would be reused by the next allocation)."""
    return ctypes.c_void_p(t.data_ptr())


def _bf(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float32)).to(torch.bfloat16).cuda()


def _f32(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float32)).cuda()


def _close(got, ref, rel):
    scale = max(np.max(np.abs(ref)), 1e-30)
    return np.max(np.abs(got - ref)) / scale <= rel


@pytest.mark.parametrize("cin,cout,act,outf", [(16, 32, 1, 0), (32, 32, 1, 0), (32, 16, 0, 1),
                                               (32, 32, 0, 0), (16, 32, 0, 0)])
@pytest.mark.parametrize("n,h,w", [(2, 32, 48), (3, 16, 16)])
def test_forward_matches_oracle(cin, cout, act, outf, n, h, w):
    """The tcgen05 forward kernel against the oracle; 16 x 16 images make the
    halo box (18 x 10 pixels) overhang the image on every side."""
    rng = np.random.default_rng(cin + cout + act + h)
    x = O.bf16(rng.standard_normal((n, h, w, cin)))
    wt = O.bf16(rng.standard_normal((cout, 9, cin)) * 0.2)
    b = rng.standard_normal(cout).astype(np.float32) * 0.1
    y = torch.empty((n, h, w, cout), dtype=torch.float32 if outf else torch.bfloat16, device="cuda")
    z = torch.empty((n, h, w, cout), dtype=torch.float32, device="cuda") if act else None
    lib = _lib()
    xd, wd, bd = _bf(x), _bf(wt), _f32(b)  # keep the buffers alive across the launch
    rc = lib.nn_conv3x3_forward(_p(xd), _p(wd), _p(bd), _p(y),
                                _p(z) if z is not None else None, n, h, w, cin, cout, act, outf, None)
    assert rc == 0
    torch.cuda.synchronize()
    zref = O.conv3x3(x, wt, b)
    if act:
        assert _close(z.cpu().numpy(), zref, 1e-5)
        yref = O.gelu(zref)
    else:
        yref = zref
    got = y.float().cpu().numpy()
    assert _close(got, yref, 1e-5 if outf else 8e-3)


@pytest.mark.parametrize("cin,cout", [(16, 32), (32, 32), (32, 16)])
def test_weight_gradient_matches_oracle(cin, cout):
    rng = np.random.default_rng(3 * cin + cout)
    n, h, w = 2, 32, 32
    x = O.bf16(rng.standard_normal((n, h, w, cin)))
    dz = O.bf16(rng.standard_normal((n, h, w, cout)))
    nblk = n * (h // 16) * (w // 16)
    partial = torch.empty(nblk * cout * 9 * cin, device="cuda")
    pdb = torch.empty(nblk * cout, device="cuda")
    dw = torch.empty((cout, 9, cin), device="cuda")
    db = torch.empty(cout, device="cuda")
    xd, dzd = _bf(x), _bf(dz)
    rc = _lib().nn_conv3x3_wgrad(_p(xd), _p(dzd), _p(partial), _p(pdb), _p(dw), _p(db), n,
                                 h, w, cin, cout, None)
    assert rc == 0
    torch.cuda.synchronize()
    dwr, dbr = O.conv3x3_wgrad(x, dz)
    assert _close(dw.cpu().numpy(), dwr, 1e-5)
    assert _close(db.cpu().numpy(), dbr, 1e-5)


def test_data_gradient_is_flipped_convolution():
    rng = np.random.default_rng(9)
    n, h, w, cin, cout = 1, 32, 32, 32, 32
    dz = O.bf16(rng.standard_normal((n, h, w, cout)))
    wt = O.bf16(rng.standard_normal((cout, 9, cin)) * 0.2)
    lib = _lib()
    wflip = torch.empty((cin, 9, cout), dtype=torch.bfloat16, device="cuda")
    wd, dzd = _bf(wt), _bf(dz)
    assert lib.nn_flip_weights(_p(wd), _p(wflip), cout, cin, None) == 0
    dx = torch.empty((n, h, w, cin), dtype=torch.bfloat16, device="cuda")
    zero = torch.zeros(cin, device="cuda")
    assert lib.nn_conv3x3_forward(_p(dzd), _p(wflip), _p(zero), _p(dx), None, n, h, w, cout,
                                  cin, 0, 0, None) == 0
    torch.cuda.synchronize()
    ref = O.conv3x3(dz, O.flip(wt))
    # the flipped convolution is the adjoint: <conv(x, w), dz> = <x, conv(dz, flip(w))>
    x = rng.standard_normal((n, h, w, cin))
    assert abs(np.sum(O.conv3x3(x, wt) * dz) - np.sum(x * ref)) < 1e-8 * np.sum(np.abs(x * ref))
    assert _close(dx.float().cpu().numpy(), ref, 8e-3)


def test_network_backward_matches_oracle():
    """Whole-network gradients (5 layers, GELU, MSE) against the oracle's
    float64 backward with the same BF16 roundings."""
    from classic_b200.corrector import ConvNet, LAYERS
    net = ConvNet(seed=1)
    rng = np.random.default_rng(2)
    n, h, w = 2, 32, 32
    x = np.zeros((n, h, w, 16))
    x[..., :8] = rng.standard_normal((n, h, w, 8))
    x = O.bf16(x)
    target = rng.standard_normal((n, h, w, 4)).astype(np.float32)
    for k in range(len(LAYERS)):  # larger last layer so every gradient is well scaled
        if k == len(LAYERS) - 1:
            net.w32[k][:4] *= 30.0
            net.w16[k].copy_(net.w32[k].to(torch.bfloat16))
    xd, td = _bf(x), _f32(target)
    pred = net.forward(xd, train=True)
    dy, loss = net.loss_grad(pred, td)
    net.backward(dy)
    torch.cuda.synchronize()
    layers = [(net.w16[k].float().cpu().numpy().astype(np.float64), net.b[k].cpu().numpy(),
               LAYERS[k][2]) for k in range(len(LAYERS))]
    out, cache = O.forward(x, layers)
    assert _close(pred.cpu().numpy(), out, 2e-2)
    lsum, g = O.mse_grad(out, target)
    assert abs(loss.item() - lsum) <= 2e-2 * lsum
    grads = O.backward(g, layers, cache)
    for k in range(len(LAYERS)):
        gw = net.gw[k].cpu().numpy()
        gb = net.gb[k].cpu().numpy()
        assert np.linalg.norm(gw - grads[k][0]) <= 5e-2 * np.linalg.norm(grads[k][0]), k
        assert np.linalg.norm(gb - grads[k][1]) <= 5e-2 * np.linalg.norm(grads[k][1]) + 1e-12, k


def test_training_fits_a_local_linear_map():
    """Adam with the device kernels learns a fixed 3x3 stencil map of the
    inputs: the loss falls by more than 10x."""
    from classic_b200.corrector import ConvNet
    rng = np.random.default_rng(4)
    n, h, w = 8, 32, 32
    x = np.zeros((n, h, w, 16))
    x[..., :8] = rng.standard_normal((n, h, w, 8))
    x = O.bf16(x)
    wtrue = rng.standard_normal((4, 9, 16)) * 0.1
    wtrue[:, :, 8:] = 0
    target = O.conv3x3(x, wtrue).astype(np.float32)
    net = ConvNet(seed=5)
    xb, tb = _bf(x), _f32(target)
    losses = []
    for it in range(300):
        pred = net.forward(xb, train=True)
        dy, loss = net.loss_grad(pred, tb)
        net.backward(dy)
        net.adam(lr=3e-3)
        losses.append(loss.item())
    assert losses[-1] < losses[0] / 10


def test_apply_correction_conserves_and_falls_back():
    lib = _lib()
    n = 32
    rng = np.random.default_rng(7)
    rho = 1.0 + 0.1 * rng.random((n, n))
    q = np.stack([rho, 0.1 * rng.standard_normal((n, n)), 0.1 * rng.standard_normal((n, n)),
                  2.5 + 0.1 * rng.random((n, n))])
    r = np.zeros((n, n, 16), dtype=np.float32)
    r[..., :4] = 0.01 * rng.standard_normal((n, n, 4))
    r[:16, :16, 0] = -50.0  # tile (0,0): density collapses -> keeps the plain step
    r[0, 0, 0] = 5000.0     # ... and its mean is not zero
    norm = np.ones(16, dtype=np.float32)
    qd = torch.as_tensor(q).cuda().contiguous()
    flags = torch.zeros(4, dtype=torch.int32, device="cuda")
    rd, nd = _f32(r), _f32(norm)
    rc = lib.nn_apply_correction(_p(qd), n, n * n, n, n, _p(rd), 16, _p(nd), 1.4, 1e-10,
                                 _p(flags), None)
    assert rc == 0
    out = qd.cpu().numpy()
    fl = flags.cpu().numpy()
    assert fl[0] == 0 and fl[1:].all()
    assert np.array_equal(out[:, :16, :16], q[:, :16, :16])
    for ty in range(2):
        for tx in range(2):
            sl = (slice(None), slice(16 * ty, 16 * ty + 16), slice(16 * tx, 16 * tx + 16))
            tot = out[sl].reshape(4, -1).sum(1) - q[sl].reshape(4, -1).sum(1)
            assert np.all(np.abs(tot) <= 1e-12 * np.abs(q[sl]).reshape(4, -1).sum(1))
    assert not np.array_equal(out[:, 16:, 16:], q[:, 16:, 16:])


def test_glue_block_average_and_features():
    lib = _lib()
    rng = np.random.default_rng(8)
    r, n = 4, 16
    fine = rng.random((4, n * r, n * r))
    fd = torch.as_tensor(fine).cuda().contiguous()
    cd = torch.empty((4, n, n), dtype=torch.float64, device="cuda")
    assert lib.nn_block_average(_p(fd), n * r, (n * r) ** 2, _p(cd), n, n * n, n, n, r, 4, None) == 0
    ref = fine.reshape(4, n, r, n, r).mean(axis=(2, 4))
    assert np.allclose(cd.cpu().numpy(), ref, rtol=1e-14, atol=0)
    qs = cd + 0.01
    norm = np.arange(16, dtype=np.float32) * 0.1 + 0.5
    x = torch.empty((1, n, n, 16), dtype=torch.bfloat16, device="cuda")
    nd = _f32(norm)
    assert lib.nn_features(_p(cd), _p(qs), n, n * n, n, n, 0, _p(nd), _p(x), None) == 0
    xs = x.float().cpu().numpy()[0]
    q = cd.cpu().numpy()
    for c in range(4):
        assert np.allclose(xs[..., c], (q[c] - norm[c]) * norm[4 + c], rtol=1e-2, atol=1e-2)
        assert np.allclose(xs[..., 4 + c], 0.01 * norm[8 + c], rtol=1e-2)
    assert np.all(xs[..., 8:] == 0)
