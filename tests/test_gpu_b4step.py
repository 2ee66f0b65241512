"""The before-step hook (b4step2, src/2d/claw2.f:626-631) on the GPU: a
device routine launched ahead of every step rewrites the annulus example's
edge velocities as the unscaled ones times cos(pi t / T), against the CPU
oracle.  The device cos() and the host's may differ in the last bit, so the
comparison is to 1e-12 relative."""
import numpy as np
import pytest

from classic_b200 import problems
from classic_b200.solver import Solver, run
from helpers import rel_diff
from pyoracle import OracleGrid, run_oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dsplit", ["unsplit", "godunov"])
def test_reversing_annulus_frames(dsplit):
    rd, solver, _, q0, aux = problems.advection_2d_annulus(mx=40, my=120, nout=4, tfinal=1.0)
    rd.clawdata.dt_max = 0.005
    rd.clawdata.dimensional_split = dsplit
    params = {"period": 1.0}
    fg = run(rd, solver, params, q0, aux, user_b4step="reversing")
    fo = run_oracle(rd, solver, params, q0, aux, user_b4step="reversing")
    assert len(fg) == len(fo)
    for a, b in zip(fg, fo):
        assert a.t == b[1]
        assert np.all(rel_diff(a.q, b[2]) <= 1e-12)
    assert np.abs(fg[-1].q - q0).max() < 0.15


def test_single_steps_use_the_step_start_time():
    rd, solver, _, q0, aux = problems.advection_2d_annulus(mx=40, my=120)
    params = {"period": 0.3}
    g = Solver(rd.clawdata, solver, params, user_b4step="reversing")
    o = OracleGrid(rd.clawdata, solver, params, user_b4step="reversing")
    for s in (g, o):
        s.set_q(q0)
        s.set_aux(aux)
    t = 0.0
    for dt in (0.004, 0.006, 0.005):
        cg, co = g.step(dt), o.step(dt, t)
        t += dt
        assert abs(cg - co) <= 1e-13 * co
        assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-12)
    g.close()
