"""1D path (single persistent CTA, whole claw1 loop in one launch) against
the oracle and, through it, the reference's regression pins."""
import json
import os

import numpy as np
import pytest

from classic_b200 import problems
from classic_b200.solver import run
from helpers import e26, same
from pyoracle import run_oracle

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "regression_sums.json")))


@pytest.mark.parametrize("builder", [problems.acoustics_1d_example1,
                                     problems.acoustics_1d_heterogeneous,
                                     problems.acoustics_1d_config])
def test_frames_bitwise(builder):
    rd, solver, params, q0, aux = builder()
    fg = run(rd, solver, params, q0, aux)
    fo = run_oracle(rd, solver, params, q0, aux)
    assert len(fg) == len(fo)
    for a, b in zip(fg, fo):
        assert a.t == b[1]
        assert same(a.q, b[2])
        if b[3]:
            assert a.stats["steps_taken"] == b[3]["steps_taken"]
            assert a.stats["dt_next"] == b[3]["dt_next"]


def test_regression_pins_on_gpu():
    rd, solver, params, q0, aux = problems.acoustics_1d_heterogeneous()
    fg = [f for f in run(rd, solver, params, q0, aux) if f.frame > 0]
    ref = GOLD["acoustics_1d_heterogeneous"]["frames"]
    for f in fg:
        sums = [float(e26(f.q[m]).sum()) for m in range(2)]
        np.testing.assert_allclose(sums, ref[str(f.frame)], rtol=1e-12)


@pytest.mark.parametrize("bc", [("wall", "wall"), ("periodic", "periodic"), ("extrap", "wall")])
@pytest.mark.parametrize("lim", ["minmod", "superbee", "vanleer", "mc", "none"])
def test_bcs_and_limiters(bc, lim):
    rd, solver, params, q0, aux = problems.acoustics_1d_example1(mx=333, nout=2, tfinal=0.7)
    rd.clawdata.bc_lower[0], rd.clawdata.bc_upper[0] = bc
    rd.clawdata.limiter = [lim, lim]
    fg = run(rd, solver, params, q0, aux)
    fo = run_oracle(rd, solver, params, q0, aux)
    for a, b in zip(fg, fo):
        assert same(a.q, b[2])
