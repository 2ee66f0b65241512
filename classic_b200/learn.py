"""Train and evaluate the learned coarse-grid corrector on the seeded 2D
Euler four-quadrant family.

    python -m classic_b200.learn --train 256 --heldout 16 --truth 4 \\
        --iters 3000 --out results.json

1. Pairs: for every training seed, coarse (n^2) / fine ((4n)^2) runs to
   t_final with the coarse Courant-number dt; K coarse steps per seed are
   kept (features and residual targets, on the device).
2. Scaling: the feature and target scales are recalibrated on the pairs.
3. Training: Adam on random 64x64 crops with this library's BF16 kernels.
4. Evaluation on held-out seeds: plain coarse, corrected coarse and plain
   fine FP64 runs to t_final; L1 errors against the block-averaged fine run
   for every held-out seed, and against a (8n)^2 plain run for the first
   --truth seeds; device times of the plain fine run and the corrected
   coarse run.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import corrector as C


def _log(*a):
    print(*a, flush=True)


def generate(seeds, norm, n, keep, rng, net=None, alpha=1.0, interval=1, fine_precision="fp64"):
    torch = C._torch()
    total = len(seeds) * keep
    x = torch.empty((total, n, n, 16), dtype=torch.bfloat16, device="cuda")
    t = torch.empty((total, n, n, 4), dtype=torch.float32, device="cuda")
    gen = C.PairGenerator(n=n)
    used = 0
    steps_all = []
    for seed in seeds:
        # the steps kept: spread over the run (90..250 coarse steps to t_final at 256^2)
        est = int(0.6 * n) // interval  # windows of `interval` coarse steps
        kept = sorted(rng.choice(np.arange(1 if interval > 1 else 2, est),
                                 size=min(keep, est - 2), replace=False).tolist())
        steps, k = gen.run(seed, norm, kept, x, t, used, net=net, alpha=alpha, interval=interval,
                           fine_precision=fine_precision)
        if k and not (torch.isfinite(x[used:used + k].float()).all() and
                      torch.isfinite(t[used:used + k]).all()):
            k = 0  # a run that left the physical states: drop its pairs
        used += k
        steps_all.append(steps)
    return x[:used], t[:used], steps_all


def recalibrate(x, t, norm):
    """Rescale features / targets to unit standard deviation per channel and
    fold the factors into the normalisation used at inference."""
    torch = C._torch()
    v = norm.values.copy()
    for c in range(8):
        s = float(x[..., c].float().std())
        if s > 0:
            x[..., c] = (x[..., c].float() / s).to(torch.bfloat16)
            v[4 + c] /= s  # channels 0..3 scale q, 4..7 the increments
    for c in range(4):
        s = float(t[..., c].std())
        if s > 0:
            t[..., c] /= s
            v[12 + c] /= s
    return C.Norm(v)


def choose_alpha(net, norm, seeds, n, alphas=(0.0, 0.25, 0.5, 0.75, 1.0), interval=1):
    """The corrector's gain alpha with the smallest mean L1 error against the
    block-averaged fine run on validation seeds (alpha = 0 is the plain
    step, so the chosen corrector is never worse than plain there)."""
    refs = {s: C.block_average(C.plain_run(s, 4 * n)[0], 4) for s in seeds}
    table = []
    for a in alphas:
        errs = []
        for s in seeds:
            if a == 0.0:
                q = C.plain_run(s, n)[0]
            else:
                q = C.corrected_run(net, norm, s, n=n, alpha=a, interval=interval)[0]
            e = C.l1_error(q, refs[s])
            errs.append(e if np.isfinite(e) else np.inf)
        table.append((a, float(np.mean(errs))))
        _log(f"alpha {a}: validation error {table[-1][1]:.5f}")
    best = min(table, key=lambda r: r[1])[0]
    return best, table


def evaluate(net, norm, seeds, n, truth_count, alpha=1.0, interval=1):
    out = []
    for k, seed in enumerate(seeds):
        qc, sc, tc = C.plain_run(seed, n)
        qk, sk, frac, tk = C.corrected_run(net, norm, seed, n=n, alpha=alpha, interval=interval)
        qf, sf, tf = C.plain_run(seed, 4 * n)
        ref = C.block_average(qf, 4)
        row = dict(seed=seed, alpha=alpha, coarse_steps=sc, fine_steps=sf, corrected_steps=sk,
                   corrected_tile_fraction=frac, fine_seconds=tf, corrected_seconds=tk,
                   coarse_seconds=tc, finite=bool(np.isfinite(qk).all() and np.isfinite(qf).all()),
                   err_vs_fine_plain=C.l1_error(qc, ref), err_vs_fine_corrected=C.l1_error(qk, ref))
        if k < truth_count:
            qt, st, tt = C.plain_run(seed, 8 * n)
            truth = C.block_average(qt, 8)
            row.update(err_truth_plain=C.l1_error(qc, truth), err_truth_corrected=C.l1_error(qk, truth),
                       err_truth_fine=C.l1_error(C.block_average(qf, 4), truth), truth_steps=st)
        out.append(row)
        _log(json.dumps(row))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--train", type=int, default=256)
    ap.add_argument("--heldout", type=int, default=16)
    ap.add_argument("--truth", type=int, default=4)
    ap.add_argument("--keep", type=int, default=16, help="coarse steps kept per training seed")
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=3e-4)
    ap.add_argument("--noise", type=float, default=0.01)
    ap.add_argument("--clip", type=float, default=5.0, help="clip targets at +-clip std")
    ap.add_argument("--validation", type=int, default=4)
    ap.add_argument("--huber", type=float, default=1.0, help="Huber delta (0: MSE)")
    ap.add_argument("--rounds", type=int, default=2,
                    help="on-policy rounds: pairs from corrected trajectories of new seeds")
    ap.add_argument("--round-seeds", type=int, default=128)
    ap.add_argument("--round-iters", type=int, default=6000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--interval", type=int, default=1,
                    help="coarse steps between corrections (windows of the pairs)")
    ap.add_argument("--fine-precision", default="fp64", choices=["fp64", "fp64_fma"],
                    help="arithmetic of the fine runs that make the training targets "
                         "(evaluation always uses the reference-order FP64 fine run)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    torch = C._torch()
    rng = np.random.default_rng(args.seed)
    train_seeds = list(range(10000, 10000 + args.train))
    held_seeds = list(range(20000, 20000 + args.heldout))
    t0 = time.perf_counter()
    K = args.interval
    x, t, steps = generate(train_seeds, C.default_norm(), args.n, args.keep, rng, interval=K,
                           fine_precision=args.fine_precision)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    _log(f"pairs: {x.shape[0]} from {len(train_seeds)} seeds in {t_gen:.1f} s "
         f"(windows of {K} coarse steps per run {min(steps)}..{max(steps)})")
    norm = recalibrate(x, t, C.default_norm())
    if args.clip > 0:
        t.clamp_(-args.clip, args.clip)  # shock residuals are heavy-tailed
    C.project_tiles(t)
    net = C.ConvNet(seed=args.seed)
    t0 = time.perf_counter()
    losses = C.train(net, x, t, iters=args.iters, batch=args.batch, lr=args.lr, seed=args.seed,
                     noise=args.noise, delta=args.huber,
                     log=lambda it, l: _log(f"iter {it} loss {l:.4e}"))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    # on-policy rounds: pairs along the corrected coarse trajectories, where
    # the network's own errors have moved the state, then more training on
    # all pairs (DAgger)
    for rnd in range(args.rounds):
        seeds_r = list(range(50000 + 1000 * rnd, 50000 + 1000 * rnd + args.round_seeds))
        xr, tr_, _ = generate(seeds_r, norm, args.n, args.keep, rng, net=net, alpha=0.5,
                              interval=K, fine_precision=args.fine_precision)
        if args.clip > 0:
            tr_.clamp_(-args.clip, args.clip)
        C.project_tiles(tr_)
        x = torch.cat([x, xr])
        t = torch.cat([t, tr_])
        del xr, tr_
        _log(f"round {rnd + 1}: {x.shape[0]} pairs")
        t1 = time.perf_counter()
        losses += C.train(net, x, t, iters=args.round_iters, batch=args.batch, lr=args.lr * 0.5,
                          seed=args.seed + rnd + 1, noise=args.noise, delta=args.huber,
                          log=lambda it, l: _log(f"round {rnd + 1} iter {it} loss {l:.4e}"))
        torch.cuda.synchronize()
        t_train += time.perf_counter() - t1
    del x, t
    # one-step skill on pairs of unseen seeds (same scaling and projection)
    xv, tv, _ = generate(list(range(40000, 40004)), C.Norm(C.default_norm().values), args.n, 4, rng,
                         interval=K)
    if xv.shape[0]:
        sc = C.default_norm().values
        for c in range(8):
            xv[..., c] = (xv[..., c].float() * float(norm.values[4 + c] / sc[4 + c])).to(torch.bfloat16)
        for c in range(4):
            tv[..., c] *= float(norm.values[12 + c] / sc[12 + c])
        if args.clip > 0:
            tv.clamp_(-args.clip, args.clip)
        C.project_tiles(tv)
        gain = C.one_step_gain(net, xv, tv)
        _log(f"one-step relative error on unseen pairs: {gain:.3f}")
    else:
        gain = float("nan")
    del xv, tv
    val_seeds = list(range(30000, 30000 + args.validation))
    alpha, table = (choose_alpha(net, norm, val_seeds, args.n, interval=K) if val_seeds
                    else (1.0, []))
    rows = evaluate(net, norm, held_seeds, args.n, args.truth, alpha=alpha, interval=K)
    good = [r for r in rows if r["finite"]]
    summary = dict(
        alpha=alpha, alpha_table=table, one_step_relative_error=gain, interval=K,
        pairs_seconds=t_gen, train_seconds=t_train, iters=args.iters, batch=args.batch,
        train_seeds=len(train_seeds), heldout_seeds=len(held_seeds), loss_first=losses[0][1],
        loss_last=losses[-1][1],
        mean_err_vs_fine_plain=float(np.mean([r["err_vs_fine_plain"] for r in good])),
        mean_err_vs_fine_corrected=float(np.mean([r["err_vs_fine_corrected"] for r in good])),
        speedup_fine_over_corrected=float(np.mean([r["fine_seconds"] / r["corrected_seconds"]
                                                  for r in good])))
    tr = [r for r in good if "err_truth_fine" in r]
    if tr:
        summary.update(
            mean_err_truth_plain=float(np.mean([r["err_truth_plain"] for r in tr])),
            mean_err_truth_corrected=float(np.mean([r["err_truth_corrected"] for r in tr])),
            mean_err_truth_fine=float(np.mean([r["err_truth_fine"] for r in tr])))
        summary["corrected_over_fine_error"] = (summary["mean_err_truth_corrected"] /
                                                summary["mean_err_truth_fine"])
    _log(json.dumps(summary))
    if args.out:
        with open(args.out, "w") as f:
            json.dump(dict(summary=summary, rows=rows, losses=losses, norm=norm.values.tolist(),
                           args=vars(args)), f, indent=1)
        C.save_trained(args.out.replace(".json", "_trained.npz"), net, norm, alpha, K)
    return summary


if __name__ == "__main__":
    main()
