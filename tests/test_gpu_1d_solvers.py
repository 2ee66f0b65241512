"""1D advection and 1D Euler (Roe with the Harten-Hyman entropy fix) on the
single-CTA 1D path, bit-identical to the oracle frame by frame, with the
dt controller's step counts and next dt."""
import numpy as np
import pytest

from classic_b200 import problems
from classic_b200.solver import run
from helpers import same
from pyoracle import run_oracle

pytestmark = pytest.mark.gpu


def _check(rd, solver, params, q0, aux=None):
    fg = run(rd, solver, params, q0, aux)
    fo = run_oracle(rd, solver, params, q0, aux)
    assert len(fg) == len(fo)
    for a, b in zip(fg, fo):
        assert a.t == b[1]
        assert same(a.q, b[2])
        if b[3]:
            assert a.stats["steps_taken"] == b[3]["steps_taken"]
            assert a.stats["dt_next"] == b[3]["dt_next"]


def test_advection_1d_example1():
    _check(*problems.advection_1d_example1())


@pytest.mark.parametrize("mx", [2000, 1000, 5000])
def test_euler_1d_wcblast(mx):
    """2000 cells (the example) and 5000 keep the interface arrays in a
    global buffer, 1000 keeps everything in shared memory."""
    _check(*problems.euler_1d_wcblast(mx=mx, nout={2000: 20, 1000: 2, 5000: 8}[mx]))


@pytest.mark.parametrize("bc", [("wall", "wall"), ("periodic", "periodic"), ("extrap", "extrap")])
@pytest.mark.parametrize("lim", ["minmod", "superbee", "vanleer", "mc", "none"])
def test_euler_1d_bcs_and_limiters(bc, lim):
    rd, solver, params, q0, aux = problems.euler_1d_wcblast(mx=257, nout=2, tfinal=0.01)
    rd.clawdata.bc_lower[0], rd.clawdata.bc_upper[0] = bc
    rd.clawdata.limiter = [lim] * 3
    _check(rd, solver, params, q0, aux)


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("u", [0.7, -1.3])
def test_advection_1d_speeds_and_orders(order, u):
    rd, solver, _, q0, aux = problems.advection_1d_example1(mx=311, nout=3, tfinal=0.5)
    rd.clawdata.order = order
    _check(rd, solver, {"u": u}, q0, aux)
