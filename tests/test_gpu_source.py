"""Source-term splitting on the GPU (src1 / src2 hooks of
src/1d/claw1.f:486-509 and src/2d/claw2.f:635-738) with the radial source of
examples/acoustics_2d_radial/1drad/src1.f, against the CPU oracle.

In 1D the source steps run inside the single-CTA time loop; in 2D they are
fused into the step kernels (Strang's first half on the values a step reads,
the second half or Godunov's whole step on the values it writes), so a
source step costs no extra pass over q.  FP64 results compare bit for bit."""
import numpy as np
import pytest

from classic_b200 import problems
from classic_b200.solver import Solver, run
from helpers import same
from pyoracle import OracleGrid, run_oracle

pytestmark = pytest.mark.gpu


def _frames_equal(fg, fo):
    assert len(fg) == len(fo)
    for a, b in zip(fg, fo):
        assert a.t == b[1]
        assert same(a.q, b[2]), f"frame {a.frame}"


@pytest.mark.parametrize("split", ["godunov", "strang"])
@pytest.mark.parametrize("order", [1, 2])
def test_1drad_example_bitwise(split, order):
    """examples/acoustics_2d_radial/1drad (2000 cells, the first dt rejected)."""
    rd, solver, params, q0, _ = problems.radial_acoustics_1d(nout=5, tfinal=0.5, order=order,
                                                             source_split=split)
    fg = run(rd, solver, params, q0, user_source="radial")
    fo = run_oracle(rd, solver, params, q0, user_source="radial")
    _frames_equal(fg, fo)


@pytest.mark.parametrize("source", ["godunov", "strang"])
@pytest.mark.parametrize("dsplit", ["unsplit", "godunov", "strang"])
def test_axisymmetric_2d_bitwise(source, dsplit):
    rd, solver, params, q0, _ = problems.axisymmetric_acoustics_2d(nr=150, nz=37, tfinal=0.2,
                                                                   source_split=source,
                                                                   split=dsplit)
    fg = run(rd, solver, params, q0, user_source="radial")
    fo = run_oracle(rd, solver, params, q0, user_source="radial")
    _frames_equal(fg, fo)


def test_axisymmetric_2d_large_bitwise():
    """Enough rows and strips for several row chunks per warp."""
    rd, solver, params, q0, _ = problems.axisymmetric_acoustics_2d(nr=500, nz=300, tfinal=0.05,
                                                                   nout=1, source_split="strang")
    fg = run(rd, solver, params, q0, user_source="radial")
    fo = run_oracle(rd, solver, params, q0, user_source="radial")
    _frames_equal(fg, fo)


def test_single_step_runs_without_the_source():
    """claw_step is step2 alone (claw2 wraps the source steps around it)."""
    rd, solver, params, q0, _ = problems.axisymmetric_acoustics_2d(nr=64, nz=16,
                                                                   source_split="strang")
    g = Solver(rd.clawdata, solver, params, user_source="radial")
    o = OracleGrid(rd.clawdata, solver, params, user_source="radial")
    g.set_q(q0)
    o.set_q(q0)
    for dt in (0.003, 0.004):
        assert g.step(dt) == o.step(dt)
        assert same(g.get_q(), o.get_q())
    g.close()
