"""Learned coarse-grid corrector for the 2D Euler step.

A coarse grid advanced by the plain wave-propagation step is nudged, after
every step, by a small convolutional network trained to predict the
difference between the block-averaged fine-grid solution and the plain
coarse step:

    q_{n+1} = S_coarse(q_n) + C(q_n, S_coarse(q_n) - q_n)

The network has five 3x3 convolutions (32 channels, GELU), 8 input channels
(4 conserved fields + the plain step's 4 increments, normalised) and 4
outputs (the residual, normalised).  Its forward and backward passes run on
the device through this library's own kernels (include/claw_nn.h, BF16
tensor-core products with FP32 accumulation); PyTorch only holds the device
buffers.  The plain solver stays the fallback: a 16x16 tile whose corrected
density or pressure is not positive, or whose conserved totals move by more
than 1e-10 relative, keeps the plain step (the correction is projected to
zero tile mean, so totals move only by rounding).

Training pairs come from this solver: per coarse step, the coarse state is
the block average of a fine run (4x finer, same seeded initial data), the
plain coarse step is taken with the coarse Courant-number dt, the fine run
advances over the same interval, and the target is the difference of the
two (one-step teacher forcing).
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _lib, problems
from ._lib import check
from .solver import Solver

# (cin, cout, act): channel counts padded to the kernels' shapes; layer 1
# uses 8 of its 16 input channels, layer 5 writes 4 of its 16 outputs
LAYERS = [(16, 32, 1), (32, 32, 1), (32, 32, 1), (32, 32, 1), (32, 16, 0)]
IN_REAL, OUT_REAL = 8, 4


def _torch():
    import torch
    return torch


def _stream():
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


class _DevView:
    """__cuda_array_interface__ over a raw device pointer (zero copy)."""

    def __init__(self, ptr, shape, strides, typestr="<f8"):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": tuple(strides)}


def q_view(solver: Solver):
    """The solver's current device q as a torch tensor [meqn][my][mx] (a view)."""
    torch = _torch()
    ptr, es, ld, fp = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong()
    check(solver.lib.claw_q_device(solver._h, ctypes.byref(ptr), ctypes.byref(es),
                                   ctypes.byref(ld), ctypes.byref(fp)), "claw_q_device")
    meqn, my, mx = solver.q_shape
    v = _DevView(ptr.value, (meqn, my, mx), (fp.value * 8, ld.value * 8, 8))
    return torch.as_tensor(v, device="cuda"), ld.value, fp.value


class ConvNet:
    """The corrector network on the device: FP32 master weights with BF16
    copies, Adam state, and the activations of the last forward pass."""

    def __init__(self, seed: int = 0):
        torch = _torch()
        self.lib = _lib.load()
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.w32, self.w16, self.b, self.m, self.v, self.gw, self.gb = [], [], [], [], [], [], []
        self.mb, self.vb = [], []
        for k, (cin, cout, act) in enumerate(LAYERS):
            fan_in = 9 * (IN_REAL if k == 0 else cin)
            std = math.sqrt(2.0 / fan_in) if act else 0.1 * math.sqrt(1.0 / fan_in)
            w = torch.randn((cout, 9, cin), generator=g) * std
            if k == 0:
                w[:, :, IN_REAL:] = 0.0
            if k == len(LAYERS) - 1:
                w[OUT_REAL:] = 0.0
            w = w.cuda()
            self.w32.append(w.contiguous())
            self.w16.append(w.to(torch.bfloat16).contiguous())
            self.b.append(torch.zeros(cout, device="cuda"))
            for lst in (self.m, self.v, self.gw):
                lst.append(torch.zeros_like(w))
            for lst in (self.mb, self.vb, self.gb):
                lst.append(torch.zeros(cout, device="cuda"))
        self.step_count = 0
        self._cache = None

    # -- device buffers sized per input shape --------------------------------
    def _buffers(self, n, h, w):
        torch = _torch()
        key = (n, h, w)
        if self._cache is not None and self._cache["key"] == key:
            return self._cache
        c = {"key": key, "acts": [], "zs": []}
        for cin, cout, act in LAYERS:
            if act:
                c["acts"].append(torch.empty((n, h, w, cout), dtype=torch.bfloat16, device="cuda"))
                c["zs"].append(torch.empty((n, h, w, cout), dtype=torch.float32, device="cuda"))
        c["out"] = torch.empty((n, h, w, LAYERS[-1][1]), dtype=torch.float32, device="cuda")
        c["dy"] = torch.empty((n, h, w, LAYERS[-1][1]), dtype=torch.bfloat16, device="cuda")
        c["d32a"] = torch.empty((n, h, w, 32), dtype=torch.bfloat16, device="cuda")
        c["d32b"] = torch.empty((n, h, w, 32), dtype=torch.bfloat16, device="cuda")
        nblk = n * (h // 16) * (w // 16)
        c["partial"] = torch.empty(nblk * 32 * 9 * 32, dtype=torch.float32, device="cuda")
        c["pdb"] = torch.empty(nblk * 32, dtype=torch.float32, device="cuda")
        c["wt"] = torch.empty(32 * 9 * 32, dtype=torch.bfloat16, device="cuda")
        c["loss"] = torch.zeros(1, dtype=torch.float64, device="cuda")
        self._cache = c
        return c

    def forward(self, x, train: bool = False):
        """x: [n][h][w][16] BF16 (device).  Returns the FP32 output
        [n][h][w][16] (4 meaningful channels)."""
        n, h, w, _ = x.shape
        c = self._buffers(n, h, w)
        st = _stream()
        a = x
        for k, (cin, cout, act) in enumerate(LAYERS):
            last = k == len(LAYERS) - 1
            y = c["out"] if last else c["acts"][k]
            z = c["zs"][k] if (train and act) else None
            check(self.lib.nn_conv3x3_forward(_p(a), _p(self.w16[k]), _p(self.b[k]), _p(y),
                                              _p(z) if z is not None else None, n, h, w, cin, cout,
                                              act, 1 if last else 0, st), "nn_conv3x3_forward")
            a = y
        c["x"] = x
        return c["out"]

    def backward(self, dy):
        """dy: d(loss)/d(output) [n][h][w][16] BF16; fills self.gw / self.gb."""
        n, h, w, _ = dy.shape
        c = self._cache
        st = _stream()
        d = dy
        for k in range(len(LAYERS) - 1, -1, -1):
            cin, cout, act = LAYERS[k]
            if act:
                dz = c["d32a"] if d is not c["d32a"] else c["d32b"]
                check(self.lib.nn_gelu_backward(_p(d), _p(c["zs"][k]), _p(dz), d.numel(), st),
                      "nn_gelu_backward")
            else:
                dz = d
            a_in = c["x"] if k == 0 else c["acts"][k - 1]
            check(self.lib.nn_conv3x3_wgrad(_p(a_in), _p(dz), _p(c["partial"]), _p(c["pdb"]),
                                            _p(self.gw[k]), _p(self.gb[k]), n, h, w, cin, cout, st),
                  "nn_conv3x3_wgrad")
            if k > 0:
                check(self.lib.nn_flip_weights(_p(self.w16[k]), _p(c["wt"]), cout, cin, st),
                      "nn_flip_weights")
                dx = c["d32b"] if dz is c["d32a"] else c["d32a"]
                check(self.lib.nn_conv3x3_forward(_p(dz), _p(c["wt"]), _p(self._zero_bias(cin)),
                                                  _p(dx), None, n, h, w, cout, cin, 0, 0, st),
                      "nn_conv3x3_forward (data gradient)")
                d = dx

    def _zero_bias(self, n):
        torch = _torch()
        if not hasattr(self, "_zb"):
            self._zb = torch.zeros(64, device="cuda")
        return self._zb

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        st = _stream()
        for k in range(len(LAYERS)):
            check(self.lib.nn_adam(_p(self.w32[k]), _p(self.gw[k]), _p(self.m[k]), _p(self.v[k]),
                                   _p(self.w16[k]), self.w32[k].numel(), lr, b1, b2, eps,
                                   self.step_count, st), "nn_adam")
            check(self.lib.nn_adam(_p(self.b[k]), _p(self.gb[k]), _p(self.mb[k]), _p(self.vb[k]),
                                   None, self.b[k].numel(), lr, b1, b2, eps, self.step_count, st),
                  "nn_adam")

    def loss_grad(self, pred, target, delta=0.0):
        """MSE (delta = 0) or Huber loss on the 4 output channels (NaN targets
        masked); returns (dy, the device loss accumulator)."""
        c = self._cache
        c["loss"].zero_()
        n, h, w, cp = pred.shape
        check(self.lib.nn_mse_grad(_p(pred), _p(target), _p(c["dy"]), _p(c["loss"]), n * h * w, cp,
                                   OUT_REAL, float(delta), _stream()), "nn_mse_grad")
        return c["dy"], c["loss"]

    def state(self):
        return {"w": [w.cpu().numpy() for w in self.w32], "b": [b.cpu().numpy() for b in self.b]}

    def load(self, state):
        torch = _torch()
        for k in range(len(LAYERS)):
            self.w32[k].copy_(torch.as_tensor(state["w"][k]))
            self.w16[k].copy_(self.w32[k].to(torch.bfloat16))
            self.b[k].copy_(torch.as_tensor(state["b"][k]))


# ---------------------------------------------------------------- data ---
@dataclass
class Norm:
    """Feature / target scaling: norm[0:4] means of q, [4:8] 1/std of q,
    [8:12] 1/std of the plain increments, [12:16] 1/std of the residuals."""
    values: np.ndarray

    def device(self):
        torch = _torch()
        return torch.as_tensor(self.values.astype(np.float32), device="cuda")


def default_norm(gamma=1.4):
    # state scales of the seeded four-quadrant family; increment and residual
    # scales of a coarse step at 256^2 (set once, from a calibration run)
    v = np.zeros(16)
    v[0:4] = [1.25, 0.0, 0.0, 2.5]
    v[4:8] = 1.0 / np.array([0.45, 0.6, 0.6, 1.6])
    v[8:12] = 1.0 / np.array([5e-3, 7e-3, 7e-3, 1.5e-2])
    v[12:16] = 1.0 / np.array([1e-3, 1.5e-3, 1.5e-3, 3e-3])
    return Norm(v)


class PairGenerator:
    """Coarse (n x n) / fine (r n x r n) pairs of one seeded instance."""

    def __init__(self, n=256, ratio=4, gamma=1.4, tfinal=0.25):
        self.n, self.r, self.gamma, self.tfinal = n, ratio, gamma, tfinal
        self.lib = _lib.load()

    def run(self, seed, norm: Norm, keep_steps, x_out, t_out, slot0, net=None, alpha=1.0,
            gamma_tol=1e-10, interval=1, fine_precision="fp64"):
        """Advance one instance to tfinal in windows of `interval` coarse
        steps; for the windows whose index is in keep_steps write features
        (the window's start state and increment) / targets (the block-averaged
        fine state minus the coarse state at the window's end) into
        x_out[slot] / t_out[slot].  Without `net` every window starts from the
        block-averaged fine state (teacher forcing).  With `net` the coarse
        grid runs its own corrected trajectory (alpha times the network at
        the end of each window), so the pairs cover the states the corrector
        meets at inference, with targets from the fine run at the same times.
        Both grids advance with the library's claw2 (device-side dt control):
        the coarse one `interval` steps per call (nv(1) = interval), the fine
        one to the time the coarse window reached.  Returns (windows, slots
        used)."""
        torch = _torch()
        n, r = self.n, self.r
        rdf, solver, params, qf0, _ = problems.euler_quadrants(n=n * r, seed=seed, gamma=self.gamma)
        rdc, _, _, _, _ = problems.euler_quadrants(n=n, seed=seed, gamma=self.gamma)
        fine = Solver(rdf.clawdata, solver, params, precision=fine_precision)
        coarse = Solver(rdc.clawdata, solver, params)
        coarse.set_steps_max(interval)
        fine.set_q(qf0)
        nd = norm.device()
        st = _stream()
        qwin = torch.empty((4, n, n), dtype=torch.float64, device="cuda")  # window start
        qfa = torch.empty((4, n, n), dtype=torch.float64, device="cuda")
        win, slot = 0, slot0
        keep = set(keep_steps)
        if net is not None:
            xin = torch.empty((1, n, n, 16), dtype=torch.bfloat16, device="cuda")
            flags = torch.empty(((n + 15) // 16) ** 2, dtype=torch.int32, device="cuda")
            va = norm.values.copy()
            va[12:16] = va[12:16] / max(alpha, 1e-30)
            nda = Norm(va).device()
            qf, ldf, fsf = q_view(fine)
            qc, ldc, fsc = q_view(coarse)
            check(self.lib.nn_block_average(_p(qf), ldf, fsf, _p(qc), ldc, fsc, n, n, r, 4, st),
                  "nn_block_average")
        t, dt, dtf = 0.0, 1e-3, 1e-3 / r
        while t < self.tfinal:
            qf, ldf, fsf = q_view(fine)
            qc, ldc, fsc = q_view(coarse)
            if net is None:
                check(self.lib.nn_block_average(_p(qf), ldf, fsf, _p(qc), ldc, fsc, n, n, r, 4, st),
                      "nn_block_average")
            qwin.copy_(qc)
            torch.cuda.current_stream().synchronize()  # the solvers' streams do not wait on torch's
            info, sc = coarse.advance(t, self.tfinal, dt)
            if info not in (0, 11):
                raise RuntimeError(f"coarse run info {info}")
            t1 = sc["t_reached"]
            info, sf = fine.advance(t, t1, dtf)
            if info != 0:
                raise RuntimeError(f"fine run info {info}")
            dtf = sf["dt_next"]
            full = sc["steps_taken"] == interval
            qs, ldc, fsc = q_view(coarse)
            qsc = qs.contiguous() if ldc != n else qs
            if full and win in keep:
                qf, ldf, fsf = q_view(fine)
                check(self.lib.nn_block_average(_p(qf), ldf, fsf, _p(qfa), n, n * n, n, n, r, 4, st),
                      "nn_block_average")
                check(self.lib.nn_features(_p(qwin), _p(qsc), n, n * n, n, n, slot, _p(nd), _p(x_out),
                                           st), "nn_features")
                check(self.lib.nn_residual_target(_p(qfa), _p(qsc), n, n * n, n, n, slot, _p(nd),
                                                  _p(t_out), st), "nn_residual_target")
                slot += 1
            if net is not None and full:
                check(self.lib.nn_features(_p(qwin), _p(qsc), n, n * n, n, n, 0, _p(nd), _p(xin), st),
                      "nn_features")
                out = net.forward(xin)
                check(self.lib.nn_apply_correction(_p(qs), ldc, fsc, n, n, _p(out), 16, _p(nda),
                                                   self.gamma, gamma_tol, _p(flags), st),
                      "nn_apply_correction")
            torch.cuda.current_stream().synchronize()
            t, dt = t1, sc["dt_next"]
            win += 1
        fine.close()
        coarse.close()
        return win, slot - slot0


def train(net: ConvNet, x, target, iters=2000, batch=16, crop=64, lr=1e-3, seed=0, log=None,
          margin=5, noise=0.0, delta=0.0):
    """Adam on random crops of the stored pairs; the loss covers each crop's
    interior (margin pixels from a crop edge inside the image are masked,
    as their zero-padded context differs from the full grid).  `noise`
    perturbs the 8 input channels (normalised units) so the network sees
    states near, not only on, the teacher-forced ones."""
    torch = _torch()
    gen = torch.Generator(device="cuda").manual_seed(seed)
    ns, h, w, _ = x.shape
    losses = []
    for it in range(iters):
        idx = torch.randint(0, ns, (batch,), device="cuda", generator=gen)
        # crops start on the 16x16 tile grid the correction is projected on
        oy = torch.randint(0, (h - crop) // 16 + 1, (batch,), device="cuda", generator=gen) * 16
        ox = torch.randint(0, (w - crop) // 16 + 1, (batch,), device="cuda", generator=gen) * 16
        ar = torch.arange(crop, device="cuda")
        yy = (oy[:, None] + ar[None, :])[:, :, None]
        xx = (ox[:, None] + ar[None, :])[:, None, :]
        xb = x[idx[:, None, None], yy, xx].contiguous()
        if noise > 0:
            pert = torch.randn(xb.shape[:-1] + (8,), device="cuda", generator=gen) * noise
            xb[..., :8] = (xb[..., :8].float() + pert).to(torch.bfloat16)
        tb = target[idx[:, None, None], yy, xx].clone()
        # interior mask: a crop edge that is not the grid edge
        mask = torch.zeros((batch, crop, crop), dtype=torch.bool, device="cuda")
        top = (oy > 0)[:, None, None] & (ar[None, :, None] < margin)
        bot = (oy + crop < h)[:, None, None] & (ar[None, :, None] >= crop - margin)
        lef = (ox > 0)[:, None, None] & (ar[None, None, :] < margin)
        rig = (ox + crop < w)[:, None, None] & (ar[None, None, :] >= crop - margin)
        mask = top | bot | lef | rig
        tb[mask] = float("nan")
        pred = net.forward(xb, train=True)
        dy, loss = net.loss_grad(pred, tb, delta)
        net.backward(dy)
        # cosine decay of the step size to 1% over the run
        net.adam(lr=lr * (0.01 + 0.99 * 0.5 * (1.0 + math.cos(math.pi * it / max(iters - 1, 1)))))
        if log is not None and (it % 100 == 0 or it == iters - 1):
            valid = (~mask).sum().item() * OUT_REAL
            losses.append((it, loss.item() / max(valid, 1)))
            log(it, losses[-1][1])
    return losses


def corrected_run(net: ConvNet, norm: Norm, seed, n=256, gamma=1.4, tfinal=0.25, tol=1e-10,
                  alpha=1.0, interval=1):
    """The corrected coarse run of one instance.  The library's claw2
    (claw_advance: device-side dt control with its rejections, dt_max and
    steps_max rules) advances `interval` accepted steps per call (nv(1) =
    interval; info 11 ends a window), then alpha times the corrector is
    applied on the device, fed the window's start state and increment: one
    host round trip per window.  Returns (q, steps, corrected tile
    fraction, wall seconds of the run with the device synchronised)."""
    if alpha != 1.0:
        v = norm.values.copy()
        v[12:16] = v[12:16] / max(alpha, 1e-30)
        norm = Norm(v)
    torch = _torch()
    lib = _lib.load()
    rd, solver, params, q0, _ = problems.euler_quadrants(n=n, seed=seed, gamma=gamma)
    s = Solver(rd.clawdata, solver, params)
    s.set_q(q0)
    s.set_steps_max(interval)
    nd = norm.device()
    st = _stream()
    x = torch.empty((1, n, n, 16), dtype=torch.bfloat16, device="cuda")
    qwin = torch.empty((4, n, n), dtype=torch.float64, device="cuda")
    flags = torch.empty(((n + 15) // 16) ** 2, dtype=torch.int32, device="cuda")
    good = torch.zeros((), dtype=torch.int64, device="cuda")
    t, dt, steps, tiles = 0.0, float(rd.clawdata.dt_initial), 0, 0
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    while t < tfinal:
        qc, ld, fs = q_view(s)
        qwin.copy_(qc)
        torch.cuda.current_stream().synchronize()  # the step stream does not wait on torch's
        info, sa = s.advance(t, tfinal, dt)
        if info not in (0, 11):
            raise RuntimeError(f"corrected run: claw_advance info {info}")
        t, dt = sa["t_reached"], sa["dt_next"]
        steps += sa["steps_taken"]
        if sa["steps_taken"] == interval:
            qs, ld, fs = q_view(s)
            qsc = qs.contiguous() if ld != n else qs
            check(lib.nn_features(_p(qwin), _p(qsc), n, n * n, n, n, 0, _p(nd), _p(x), st),
                  "nn_features")
            out = net.forward(x)
            check(lib.nn_apply_correction(_p(qs), ld, fs, n, n, _p(out), 16, _p(nd), gamma, tol,
                                          _p(flags), st), "nn_apply_correction")
            good += flags.sum()
            tiles += flags.numel()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    q = s.get_q()
    s.close()
    return q, steps, good.item() / max(tiles, 1), wall


def plain_run(seed, n, gamma=1.4, tfinal=0.25, precision="fp64"):
    """The plain run of one instance (claw2's device-side dt control);
    returns (q, steps, wall seconds of the advance with the device
    synchronised, as corrected_run measures)."""
    torch = _torch()
    rd, solver, params, q0, _ = problems.euler_quadrants(n=n, seed=seed, gamma=gamma)
    s = Solver(rd.clawdata, solver, params, precision=precision)
    s.set_q(q0)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    info, st = s.advance(0.0, tfinal, float(rd.clawdata.dt_initial))
    wall = time.perf_counter() - w0
    q = s.get_q()
    s.close()
    return q, st["steps_taken"], wall


def save_trained(path, net: ConvNet, norm: Norm, alpha: float, interval: int):
    """One .npz with everything a corrected run needs: the FP32 master
    weights and biases of the five layers, the feature / target scaling, the
    chosen correction strength alpha and the correction interval."""
    st = net.state()
    np.savez(path, **{f"w{k}": w for k, w in enumerate(st["w"])},
             **{f"b{k}": b for k, b in enumerate(st["b"])},
             norm=norm.values, alpha=np.float64(alpha), interval=np.int64(interval))


def load_trained(path):
    """(net, norm, alpha, interval) from a file written by save_trained."""
    d = np.load(path)
    net = ConvNet(seed=0)
    net.load({"w": [d[f"w{k}"] for k in range(len(LAYERS))],
              "b": [d[f"b{k}"] for k in range(len(LAYERS))]})
    return net, Norm(np.array(d["norm"], dtype=np.float64)), float(d["alpha"]), int(d["interval"])


def block_average(q, r):
    m, h, w = q.shape
    return q.reshape(m, h // r, r, w // r, r).mean(axis=(2, 4))


def l1_error(q, ref):
    """Mean absolute difference per field, scaled by the field's mean
    magnitude, averaged over the four fields."""
    return float(np.mean([np.mean(np.abs(q[c] - ref[c])) / max(np.mean(np.abs(ref[c])), 1e-12)
                          for c in range(q.shape[0])]))


def project_tiles(t, tile=16):
    """Subtract each 16x16 tile's mean from the targets [n][h][w][c] (in
    place): the correction the network learns is the one applied, which keeps
    every tile's conserved totals."""
    n, h, w, c = t.shape
    v = t.view(n, h // tile, tile, w // tile, tile, c)
    v -= v.mean(dim=(2, 4), keepdim=True)
    return t


def one_step_gain(net, x, t, batch=8):
    """Relative L2 error of the network's prediction of the held-out targets
    (1 = no better than predicting zero)."""
    torch = _torch()
    num = den = 0.0
    for k in range(0, x.shape[0], batch):
        pred = net.forward(x[k:k + batch].contiguous())[..., :OUT_REAL]
        tt = t[k:k + batch]
        num += float(((pred - tt) ** 2).sum())
        den += float((tt ** 2).sum())
    return math.sqrt(num / max(den, 1e-300))
