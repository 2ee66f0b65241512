"""Time to an L1 error: what each precision buys on the 2D radial acoustics
workload (rho = 1, K = 4 on [-1, 1]^2, MC, transverse 2, to t = 0.6).

The truth is the same problem at a finer grid, in the contracted FP64 build
(within 1e-12 of the reference order), block-averaged onto each coarser grid
(the grids nest: n divides the truth's cell count).  Each row is one run from
t = 0 to t_final through claw2's dt control (one claw_advance call, the
initial dt of the workload, so the first step is rejected and retried as the
reference does): its device time (CUDA events around the launches), its wall
time (the call and the read of q) and the L1 norm of the pressure error,
dx dy sum |p - p_truth|, with the velocities' beside it.

The reference's accuracy is the reference-order FP64 row; the others show
what the contracted FP64 and the FP32 update paths cost in accuracy (nothing
visible: the discretisation error is orders of magnitude above rounding) and
save in time.

For the batched Euler ensemble the accuracy is that of claw2 on each instance
alone (the batch's results are those of one claw2 call per instance), so its
row is the time to the same solutions: `ensemble_batched_vs_serial`."""
from __future__ import annotations

import time

import numpy as np

from . import problems
from .solver import BatchSolver, Solver


def block_average(q: np.ndarray, r: int) -> np.ndarray:
    """Mean over r x r blocks of each field of q[m][ny][nx]."""
    m, h, w = q.shape
    return q.reshape(m, h // r, r, w // r, r).mean(axis=(2, 4))


def l1_norms(q: np.ndarray, ref: np.ndarray, dx: float, dy: float) -> list[float]:
    """dx dy sum |q - ref| per field."""
    return [float(dx * dy * np.sum(np.abs(q[c] - ref[c]))) for c in range(q.shape[0])]


def _run(n: int, precision: str, tfinal: float):
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=n, tfinal=tfinal)
    dt0 = float(rd.clawdata.dt_initial)
    s = Solver(rd.clawdata, solver, params, precision=precision)
    try:
        s.set_q(q0)
        s.advance(0.0, min(0.01, tfinal), dt0)  # warm-up: first launches, graph build
        s.set_q(q0)
        t0 = time.perf_counter()
        info, st = s.advance(0.0, tfinal, dt0)
        q = s.get_q()
        wall = time.perf_counter() - t0
    finally:
        s.close()
    if info != 0:
        raise RuntimeError(f"claw advance returned info={info} at n={n} ({precision})")
    return q, st, wall


def radial_time_to_l1(sizes=(512, 1024, 2048), precisions=("fp64", "fp64_fma", "fp32"),
                      truth_n: int = 4096, tfinal: float = 0.6) -> dict:
    """Rows of (n, precision, steps, device ms, wall ms, L1 of p, u, v) against
    the truth run at truth_n^2."""
    truth, tst, twall = _run(truth_n, "fp64_fma", tfinal)
    rows = []
    for n in sizes:
        if truth_n % n:
            raise ValueError(f"{n} does not divide the truth grid {truth_n}")
        ref = block_average(truth, truth_n // n)
        d = 2.0 / n
        for prec in precisions:
            q, st, wall = _run(n, prec, tfinal)
            l1 = l1_norms(q, ref, d, d)
            rows.append({"n": n, "precision": prec, "steps": st["steps_taken"],
                         "device_ms": st["device_ms"], "wall_ms": wall * 1e3,
                         "l1_p": l1[0], "l1_u": l1[1], "l1_v": l1[2]})
    return {"truth": {"n": truth_n, "precision": "fp64_fma", "steps": tst["steps_taken"],
                      "device_ms": tst["device_ms"], "wall_ms": twall * 1e3},
            "t_final": tfinal, "rows": rows}


def ensemble_batched_vs_serial(count: int = 32, precision: str = "fp64", tfinal: float = 0.25) -> dict:
    """The first `count` instances of the batched Euler workload (sides
    log-uniform in 128..1024, four-quadrant data of seeds 1000 + k) advanced
    to t_final once as one batch and once as one claw2 call per instance on
    its own handle, as the reference runs them.  Returns both times and the
    largest difference between the two sets of solutions (0 in the
    reference-order build: the batch takes each instance's own dt sequence)."""
    sizes = problems.euler_ensemble_sizes(256, seed=0)[:count]
    insts = [problems.euler_quadrants(n=n, seed=1000 + k) for k, n in enumerate(sizes)]
    # warm-up of both paths (module loading, first launches) on a short run
    w = BatchSolver([i[0] for i in insts[:2]], "euler_roe_2d", {"gamma": 1.4}, precision=precision)
    for k in range(2):
        w.set_q(k, insts[k][3])
    w.advance(0.0, 0.005)
    w.close()
    w = Solver(insts[0][0].clawdata, insts[0][1], insts[0][2], precision=precision)
    w.set_q(insts[0][3])
    w.advance(0.0, 0.005, float(insts[0][0].clawdata.dt_initial))
    w.close()
    b = BatchSolver([i[0] for i in insts], "euler_roe_2d", {"gamma": 1.4}, precision=precision)
    try:
        for k, inst in enumerate(insts):
            b.set_q(k, inst[3])
        t0 = time.perf_counter()
        info_b, st_b = b.advance(0.0, tfinal)
        qb = [b.get_q(k) for k in range(count)]
        wall_b = time.perf_counter() - t0
    finally:
        b.close()
    wall_s = dev_s = 0.0
    worst = 0.0
    identical = True
    for k, (rd, solver, params, q0, _) in enumerate(insts):
        s = Solver(rd.clawdata, solver, params, precision=precision)
        try:
            s.set_q(q0)
            t0 = time.perf_counter()
            info, st = s.advance(0.0, tfinal, float(rd.clawdata.dt_initial))
            q = s.get_q()
            wall_s += time.perf_counter() - t0
            dev_s += st["device_ms"] * 1e-3
        finally:
            s.close()
        identical = identical and np.array_equal(q, qb[k], equal_nan=True)
        fin = np.isfinite(q) & np.isfinite(qb[k])
        if fin.any():
            worst = max(worst, float(np.max(np.abs(q[fin] - qb[k][fin]))))
    updates = sum(n * n * (x["steps_taken"] + x["steps_rejected"]) for n, x in zip(sizes, st_b))
    return {"instances": count, "precision": precision, "cell_updates": updates,
            "batched": {"device_ms": st_b[0]["device_ms"], "wall_ms": wall_b * 1e3},
            "serial": {"device_ms": dev_s * 1e3, "wall_ms": wall_s * 1e3},
            "identical": identical, "max_abs_diff": worst}
