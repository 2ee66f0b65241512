"""Run a few steps of the 2D radial acoustics workload (for profiler captures).

    python -m classic_b200.profile_step --n 3072 --steps 4 --precision fp64_fma

Each step is one claw_step (bc2 + step2) of fixed dt = 0.9 dx / c.
"""
import argparse

from . import problems
from .solver import Solver


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=3072)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--precision", default="fp64_fma", choices=["fp64", "fp64_fma", "fp32"])
    args = ap.parse_args()
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=args.n)
    s = Solver(rd.clawdata, solver, params, precision=args.precision)
    s.set_q(q0)
    dt = 0.9 * (2.0 / args.n) / 2.0
    for _ in range(args.steps):
        s.step(dt)
    print(f"{args.steps} steps of {args.n}^2 ({args.precision}), sum p = {s.get_q()[0].sum():.12e}")
    s.close()


if __name__ == "__main__":
    main()
