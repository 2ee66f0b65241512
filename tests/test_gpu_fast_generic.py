"""The contracted builds (precision "fp64_fma") against the CPU restatement:
the characteristic-variable kernel for constant-coefficient acoustics (every
order, transverse_waves and pair of limiters), and the generic kernel and the
batch for the rest (other solvers, capacity).

This build contracts multiplies and adds into FMAs and replaces IEEE division
and sqrt by Newton-refined reciprocals and roots (about an ulp), so it is not
bit-identical to the reference order.  The bars:
  * linear solvers (acoustics, advection with capacity): Courant numbers
    equal to 1e-14 relative, q within 1e-12 relative per field;
  * Euler (Roe with the entropy fix; wave speeds from Newton square roots):
    Courant numbers to 1e-13, q within 1e-10 relative per field over tens of
    steps, the same step counts under claw2's dt control.
"""
import numpy as np
import pytest

from classic_b200 import problems
from classic_b200.solver import BatchSolver, Solver
from helpers import rel_diff
from pyoracle import OracleGrid

pytestmark = pytest.mark.gpu


def _pair(rd, solver, params, q0, aux=None):
    g = Solver(rd.clawdata, solver, params, precision="fp64_fma")
    o = OracleGrid(rd.clawdata, solver, params)
    g.set_q(q0)
    o.set_q(q0)
    if aux is not None:
        g.set_aux(aux)
        o.set_aux(aux)
    return g, o


@pytest.mark.parametrize("lim", ["minmod", "superbee", "vanleer", "mc", ("mc", "vanleer"),
                                 ("superbee", "minmod"), ("vanleer", "mc"), ("minmod", "superbee"),
                                 ("none", "superbee"), ("minmod", 5)])
@pytest.mark.parametrize("order,trans", [(1, 0), (1, 1), (2, 1), (2, 0), (2, 2)])
@pytest.mark.parametrize("bc", [("wall", "extrap", "periodic", "periodic"), ("extrap",) * 4,
                                ("periodic", "periodic", "wall", "wall")])
def test_acoustics_fast(lim, order, trans, bc):
    """The characteristic kernel, with one limiter compiled in (minmod,
    superbee, van Leer, MC), a pair of them compiled in (transverse 2), or the
    limiters read at run time (pairs at transverse 0 and 1, none and
    Beam-Warming)."""
    rd, solver, params, q0, _ = problems.random_acoustics_2d(
        45, 38, seed=9, limiter="mc", order=order, trans=trans, bc=bc)
    rd.clawdata.limiter = list(lim) if isinstance(lim, tuple) else [lim, lim]
    g, o = _pair(rd, solver, params, q0)
    for _ in range(20):
        cg, co = g.step(0.004), o.step(0.004)
        assert abs(cg - co) <= 1e-14 * co
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-12)
    g.close()


def test_annulus_capacity_fast():
    rd, solver, params, q0, aux = problems.advection_2d_annulus()
    g, o = _pair(rd, solver, params, q0, aux)
    ig, sg = g.advance(0.0, 0.25, float(rd.clawdata.dt_initial))
    io, so = o.advance(0.0, 0.25, float(rd.clawdata.dt_initial))
    assert ig == io == 0
    assert sg["steps_taken"] == so["steps_taken"]
    assert abs(sg["cfl_max_seen"] - so["cfl_max_seen"]) <= 1e-13 * so["cfl_max_seen"]
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-12)
    g.close()


@pytest.mark.parametrize("lim", ["mc", "vanleer", "superbee"])
@pytest.mark.parametrize("bc", [("extrap",) * 4, ("wall", "extrap", "periodic", "periodic")])
def test_euler_fast_steps(lim, bc):
    rd, solver, params, q0, _ = problems.euler_quadrants(shape=(64, 48), seed=21, limiter=lim, bc=bc)
    g, o = _pair(rd, solver, params, q0)
    for _ in range(30):
        cg, co = g.step(0.002), o.step(0.002)
        assert abs(cg - co) <= 1e-13 * co
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-10)
    g.close()


def test_euler_fast_advance():
    rd, solver, params, q0, _ = problems.euler_quadrants(n=128, seed=4)
    g, o = _pair(rd, solver, params, q0)
    ig, sg = g.advance(0.0, 0.1, float(rd.clawdata.dt_initial))
    io, so = o.advance(0.0, 0.1, float(rd.clawdata.dt_initial))
    assert ig == io == 0
    assert sg["steps_taken"] == so["steps_taken"] and sg["steps_taken"] > 20
    assert abs(sg["t_reached"] - so["t_reached"]) <= 1e-15
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-10)
    g.close()


def test_euler_batch_fast_per_instance():
    """The contracted ensemble kernel: each instance of an uneven batch against
    claw2 on it alone (the CPU restatement)."""
    sizes = [40, 23, 57, 64, 29, 45, 33, 50]
    insts = [problems.euler_quadrants(n=n, seed=100 + k) for k, n in enumerate(sizes)]
    b = BatchSolver([i[0] for i in insts], "euler_roe_2d", {"gamma": 1.4}, precision="fp64_fma")
    for k, inst in enumerate(insts):
        b.set_q(k, inst[3])
    info, stats = b.advance(0.0, 0.25)
    worst = 0.0
    for k, (rd, solver, params, q0, _) in enumerate(insts):
        o = OracleGrid(rd.clawdata, solver, params)
        o.set_q(q0)
        io, so = o.advance(0.0, 0.25, rd.clawdata.dt_initial)
        assert stats[k]["steps_taken"] == so["steps_taken"], k
        q, qo = b.get_q(k), o.get_q()
        if np.all(np.isfinite(qo)):
            d = float(np.max(rel_diff(q, qo)))
            worst = max(worst, d)
            assert d <= 1e-10, (k, d)
    b.close()
    print(f"worst relative difference over the batch: {worst:.3e}")
