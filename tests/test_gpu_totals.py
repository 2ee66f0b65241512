"""Conserved totals (claw_totals): FP64 compensated sums of capa * q over the
interior cells, formed on the device whatever the storage precision.  With
periodic boundaries the wave-propagation update is conservative, so the FP64
path keeps every total to 1e-13 relative over a run; the FP32 path's totals
are still summed in FP64 and its drift is reported against the FP64 run."""
import math

import numpy as np
import pytest

from classic_b200 import problems
from classic_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _fsum_fields(q, capa=None):
    w = np.ones_like(q[0]) if capa is None else capa
    return np.array([math.fsum((w * q[m]).ravel()) for m in range(q.shape[0])])


def _rel(a, b, scale):
    return np.abs(a - b) / scale


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_totals_match_exact_sums(precision):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(123, 77, seed=3)
    s = Solver(rd.clawdata, solver, params, precision)
    s.set_q(q0)
    tot = s.totals()
    q = s.get_q()
    exact = _fsum_fields(q)
    assert np.all(_rel(tot, exact, np.abs(q).sum(axis=(1, 2))) <= 1e-15)
    s.close()


def test_totals_with_capacity():
    rd, solver, params, q0, aux = problems.advection_2d_annulus()
    s = Solver(rd.clawdata, solver, params)
    s.set_q(q0)
    s.set_aux(aux)
    capa = aux[2][2:-2, 2:-2]
    exact = _fsum_fields(s.get_q(), capa)
    tot = s.totals()
    assert abs(tot[0] - exact[0]) <= 1e-15 * np.abs(capa * q0[0]).sum()
    s.close()


@pytest.mark.parametrize("solver_case", ["acoustics", "euler", "acoustics_split"])
def test_periodic_fp64_run_conserves_to_1e13(solver_case):
    if solver_case == "euler":
        rd, solver, params, q0, _ = problems.euler_quadrants(n=128, seed=5, bc=("periodic",) * 4)
        t1, dt0 = 0.05, 1e-3
    else:
        rd, solver, params, q0, _ = problems.random_acoustics_2d(160, 96, seed=2,
                                                                bc=("periodic",) * 4)
        t1, dt0 = 0.1, 0.005
        if solver_case == "acoustics_split":
            rd.clawdata.dimensional_split = "godunov"
    s = Solver(rd.clawdata, solver, params)
    s.set_q(q0)
    before = s.totals()
    info, st = s.advance(0.0, t1, dt0)
    assert info == 0 and st["steps_taken"] > 5
    after = s.totals()
    scale = np.abs(s.get_q()).sum(axis=(1, 2))
    assert np.all(_rel(after, before, scale) <= 1e-13), (before, after)
    s.close()


def test_3d_periodic_fp64_conserves_to_1e13():
    """Homogeneous medium: variable-coefficient acoustics in fluctuation form
    is not conservative where Z and c vary."""
    rd, solver, params, q0, aux = problems.random_acoustics_3d(24, 20, 18, seed=4,
                                                               bc=("periodic",) * 6)
    aux = np.ascontiguousarray(np.broadcast_to(aux[:, :1, :1, :1], aux.shape))
    s = Solver(rd.clawdata, solver, params)
    s.set_q(q0)
    s.set_aux(aux)
    before = s.totals()
    info, st = s.advance(0.0, 0.05, 0.01)
    assert info == 0
    after = s.totals()
    scale = np.abs(s.get_q()).sum(axis=(1, 2, 3))
    assert np.all(_rel(after, before, scale) <= 1e-13)
    s.close()


def test_fp32_drift_is_stated_against_fp64():
    rd, solver, params, q0, _ = problems.random_acoustics_2d(160, 96, seed=2, bc=("periodic",) * 4)
    drifts = {}
    for prec in ("fp64", "fp32"):
        s = Solver(rd.clawdata, solver, params, prec)
        s.set_q(q0)
        before = s.totals()
        s.advance(0.0, 0.1, 0.005)
        scale = np.abs(s.get_q()).sum(axis=(1, 2))
        drifts[prec] = float(np.max(_rel(s.totals(), before, scale)))
        s.close()
    assert drifts["fp64"] <= 1e-13
    assert drifts["fp32"] <= 1e-5  # FP32 rounding of the update, summed exactly in FP64
