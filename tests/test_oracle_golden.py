"""The CPU oracle against the reference's own regression data
(examples/*/regression_data, committed as tests/golden/regression_sums.json).
The sums are plain per-field sums over interior cells of the frame values
written with e26.16 after out2's flush of |q| < 1e-99."""
import json
import os

import numpy as np
import pytest

from classic_b200 import problems
from helpers import frame_sum
from pyoracle import run_oracle

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "regression_sums.json")))


def _sums(fn, name):
    rd, solver, params, q0, aux = fn()
    frames = [f for f in run_oracle(rd, solver, params, q0, aux) if f[0] > 0]
    out = {}
    for k, t, q, st in frames:
        out[k] = [frame_sum(q[m]) for m in range(q.shape[0])]
    return out


def test_acoustics_1d_example1_pin():
    got = _sums(problems.acoustics_1d_example1, "acoustics_1d_example1")
    ref = GOLD["acoustics_1d_example1"]["frames"]
    # frame 1 (t=0.5): the right- and left-going halves of the pulse
    np.testing.assert_allclose(got[1], ref["1"], rtol=1e-13)
    # frame 2 (t=1.0): the pulse has left through the extrapolation boundary;
    # both sums are roundoff residue, 1e-33 of frame 1's scale
    assert np.all(np.abs(got[2]) < 1e-13 * abs(ref["1"][0]))
    assert np.all(np.abs(ref["2"]) < 1e-13 * abs(ref["1"][0]))


def test_acoustics_1d_heterogeneous_pin():
    got = _sums(problems.acoustics_1d_heterogeneous, "acoustics_1d_heterogeneous")
    ref = GOLD["acoustics_1d_heterogeneous"]["frames"]
    np.testing.assert_allclose(got[1], ref["1"], rtol=1e-14)
    np.testing.assert_allclose(got[2], ref["2"], rtol=1e-12)


def test_advection_2d_annulus_pin():
    """Only 2D pin of the reference (capacity + transverse + periodic).  The
    pinned sums are ~1e-14 / 1e-12 by the +/- symmetry of the data, so they
    pin magnitude, not digits; conservation is checked exactly below."""
    got = _sums(problems.advection_2d_annulus, "advection_2d_annulus")
    ref = GOLD["advection_2d_annulus"]["frames"]
    for k in (1, 2):
        assert abs(got[k][0]) < 10 * abs(ref[str(k)][0]) + 1e-13


def test_annulus_conserves_capacity_weighted_mass():
    rd, solver, params, q0, aux = problems.advection_2d_annulus()
    frames = run_oracle(rd, solver, params, q0, aux, flush_tiny=False)
    capa = aux[2, 2:-2, 2:-2]
    m0 = np.sum(capa * q0[0])
    scale = np.sum(capa * np.abs(q0[0]))
    for k, t, q, st in frames[1:]:
        assert abs(np.sum(capa * q[0]) - m0) < 1e-13 * scale


def test_1d_pulse_splits_into_halves():
    """Known answer: the Gaussian splits into two halves of mass
    sqrt(pi/beta)/2/dx each, with u = -p/Z on the left-going half."""
    rd, solver, params, q0, aux = problems.acoustics_1d_example1(nout=2, tfinal=0.5)
    frames = run_oracle(rd, solver, params, q0, aux)
    q = frames[-1][2]
    dx = 2.0 / 400
    half = 0.5 * np.sqrt(np.pi / 200.0) / dx
    x = -1 + (np.arange(400) + 0.5) * dx
    left = x < 0.3
    np.testing.assert_allclose(q[0][left].sum(), half, rtol=1e-6)
    np.testing.assert_allclose(q[1][left].sum(), -half / 2.0, rtol=1e-6)


def test_oracle_step_is_deterministic():
    rd, solver, params, q0, aux = problems.random_acoustics_2d(17, 11, seed=3)
    from pyoracle import OracleGrid
    a = OracleGrid(rd.clawdata, solver, params)
    b = OracleGrid(rd.clawdata, solver, params)
    a.set_q(q0)
    b.set_q(q0)
    ca, cb = a.step(0.01), b.step(0.01)
    assert ca == cb and np.array_equal(a.get_q(), b.get_q())


def test_claw2_info_codes():
    from pyoracle import OracleGrid
    rd, solver, params, q0, aux = problems.random_acoustics_2d(8, 8)
    cd = rd.clawdata
    cd.cfl_desired, cd.cfl_max = 1.0, 0.9
    g = OracleGrid(cd, solver, params)
    g.set_q(q0)
    assert g.advance(0.0, 0.1, 0.01)[0] == 3
    cd.cfl_desired, cd.cfl_max = 0.9, 1.0
    cd.dt_variable = False
    g = OracleGrid(cd, solver, params)
    g.set_q(q0)
    assert g.advance(0.0, 0.1, 0.03)[0] == 2  # 0.03 does not divide 0.1
    assert g.advance(0.0, 0.2, 0.2)[0] == 12  # fixed dt, Courant number 1.6 > cfl_max


def test_acoustics_3d_heterogeneous_pin():
    """step3/flux3 with (2,22) corner transport, vc-acoustics rpn3/rpt3/rptt3,
    claw3's dt control and the piston user BC: all six pinned sums equal,
    including the roundoff-level velocity sums, which depend on every bit
    of the frame."""
    got = _sums(problems.acoustics_3d_heterogeneous, "acoustics_3d_heterogeneous")
    ref = GOLD["acoustics_3d_heterogeneous"]["frames"]
    for k in (1, 2):
        assert got[k][:3] == ref[str(k)], (k, got[k], ref[str(k)])
