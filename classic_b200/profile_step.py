"""Run a few steps of the 2D radial or 3D heterogeneous acoustics workload
(for profiler captures).

    python -m classic_b200.profile_step --n 3072 --steps 4 --precision fp64_fma
    python -m classic_b200.profile_step --dim 3 --n 128 --steps 2
    python -m classic_b200.profile_step --n 2048 --split godunov --precision fp64
    python -m classic_b200.profile_step --nn --n 256 --steps 3
    python -m classic_b200.profile_step --batch 16 --n 512 --steps 3 --precision fp64_fma
    python -m classic_b200.profile_step --n 3072 --limiter mc vanleer --transverse 1
    python -m classic_b200.profile_step --euler --n 2048 --steps 3 --precision fp64

--limiter takes one name (both waves) or two (wave 1, wave 2); --transverse
sets transverse_waves (2D).

With --euler each step is one claw_step of a single seeded four-quadrant Euler
grid (seed 7, the generic kernel) at fixed dt = 0.6 dx / max(|u| + c) of the
initial data.

With --batch K each step is one launch of the batched Euler ensemble kernel
over K seeded four-quadrant instances of n^2 cells (one claw_batch_advance
over `steps` time steps).

With --nn each step is one forward pass of the corrector network (five
tcgen05 convolutions) on a batch of 8 random n x n inputs.

Each step is one claw_step (bc + step2 / step3, or the dimensionally split
step with --split) of fixed dt = 0.9 dx / c_max.
"""
import argparse

from . import problems
from .solver import Solver


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dim", type=int, default=2, choices=[2, 3])
    ap.add_argument("--n", type=int, default=3072)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--precision", default="fp64_fma", choices=["fp64", "fp64_fma", "fp32"])
    ap.add_argument("--split", default="unsplit", choices=["unsplit", "godunov", "strang"])
    ap.add_argument("--nn", action="store_true", help="the corrector network's forward pass")
    ap.add_argument("--batch", type=int, default=0, help="Euler ensemble of this many instances")
    ap.add_argument("--euler", action="store_true", help="one four-quadrant Euler grid")
    ap.add_argument("--limiter", nargs="+", default=None,
                    help="limiter name for both waves, or one per wave")
    ap.add_argument("--transverse", type=int, default=2, choices=[0, 1, 2])
    args = ap.parse_args()
    if args.limiter is not None and len(args.limiter) not in (1, 2):
        ap.error("--limiter takes one or two names")
    if args.euler:
        import numpy as np
        rd, solver, params, q0, aux = problems.euler_quadrants(n=args.n, seed=7)
        gamma = float(params["gamma"])
        rho, mu, mv, en = (np.asarray(q0[k], dtype=np.float64) for k in range(4))
        u, v = mu / rho, mv / rho
        p = (gamma - 1.0) * (en - 0.5 * rho * (u * u + v * v))
        c = np.sqrt(gamma * p / rho)
        smax = float(np.max(np.maximum(np.abs(u), np.abs(v)) + c))
        s = Solver(rd.clawdata, solver, params, precision=args.precision)
        s.set_q(q0)
        dt = 0.6 * (1.0 / args.n) / smax
        for _ in range(args.steps):
            s.step(dt)
        print(f"{args.steps} Euler steps of {args.n}^2 ({args.precision}), "
              f"sum rho = {s.get_q()[0].sum():.12e}")
        s.close()
        return
    if args.batch:
        from .solver import BatchSolver
        insts = [problems.euler_quadrants(n=args.n, seed=1000 + k) for k in range(args.batch)]
        prec = "fp64_fma" if args.precision == "fp64_fma" else "fp64"
        b = BatchSolver([i[0] for i in insts], "euler_roe_2d", {"gamma": 1.4}, precision=prec)
        for k, inst in enumerate(insts):
            b.set_q(k, inst[3])
        dt = 1e-3 * 256 / args.n
        b.advance(0.0, args.steps * dt, [dt] * args.batch)  # one launch per step
        print(f"{args.steps} ensemble steps of {args.batch} x {args.n}^2 ({prec}), "
              f"sum rho = {sum(float(b.get_q(k)[0].sum()) for k in range(args.batch)):.12e}")
        b.close()
        return
    if args.nn:
        import torch

        from .corrector import ConvNet
        net = ConvNet(seed=0)
        x = torch.randn((8, args.n, args.n, 16), device="cuda").to(torch.bfloat16)
        for _ in range(args.steps):
            y = net.forward(x)
        torch.cuda.synchronize()
        print(f"{args.steps} forward passes of 8 x {args.n}^2, sum = {float(y.float().sum()):.6e}")
        return
    if args.dim == 2:
        rd, solver, params, q0, aux = problems.radial_acoustics_2d(n=args.n)
        cmax = 2.0
        prec = args.precision
    else:
        rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=args.n)
        cmax = 1.0
        prec = args.precision
    rd.clawdata.dimensional_split = args.split
    if args.limiter is not None:
        lims = args.limiter if len(args.limiter) == 2 else args.limiter * 2
        rd.clawdata.limiter = lims
    if args.dim == 2:
        rd.clawdata.transverse_waves = args.transverse
    s = Solver(rd.clawdata, solver, params, precision=prec)
    s.set_q(q0)
    if aux is not None:
        s.set_aux(aux)
    dt = 0.9 * (2.0 / args.n) / cmax
    for _ in range(args.steps):
        s.step(dt)
    print(f"{args.steps} steps of {args.n}^{args.dim} ({prec}, {args.split}), "
          f"sum p = {s.get_q()[0].sum():.12e}")
    s.close()


if __name__ == "__main__":
    main()
