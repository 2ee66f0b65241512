"""The threaded timing variant of the CPU restatement (the CPU baseline on
all host cores).  3D: blocks of one colour run in parallel as step3.f90 runs
them under OpenMP, so every cell gets its contributions in the serial order
and the threaded step equals the serial one bit for bit.  2D: every third
slice runs in parallel (the reference's 2D step is serial), which reorders
each cell's sums: equal to roundoff."""
import numpy as np

from classic_b200 import problems
from helpers import rel_diff
from pyoracle import OracleGrid


def _steps(rd, solver, params, q0, aux, threads, dt, n):
    g = OracleGrid(rd.clawdata, solver, params, variant="fast")
    g.lib.orc_set_threads(threads)
    try:
        g.set_q(q0)
        if aux is not None:
            g.set_aux(aux)
        cfl = [g.step(dt) for _ in range(n)]
        return g.get_q(), cfl
    finally:
        g.lib.orc_set_threads(1)


def test_threaded_3d_step_is_bitwise_serial():
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=14)
    qa, ca = _steps(rd, solver, params, q0, aux, 1, 0.02, 3)
    qb, cb = _steps(rd, solver, params, q0, aux, 4, 0.02, 3)
    assert ca == cb
    assert np.array_equal(qa, qb)


def test_threaded_2d_step_matches_serial():
    rd, solver, params, q0, _ = problems.random_acoustics_2d(53, 41, seed=3)
    qa, ca = _steps(rd, solver, params, q0, None, 1, 0.004, 3)
    qb, cb = _steps(rd, solver, params, q0, None, 3, 0.004, 3)
    assert ca == cb
    assert np.all(rel_diff(qb, qa) < 1e-13)
