"""Source-term splitting in the CPU oracle (src1 / src2 hooks of
src/1d/claw1.f:486-509 and src/2d/claw2.f:635-738) with the radial source of
examples/acoustics_2d_radial/1drad/src1.f.

Known answer: the 2D radial example (examples/acoustics_2d_radial, a
Cartesian grid) and its 1drad companion (the same pulse in the radius with
the geometric source) describe the same cylindrically symmetric field, so the
2D solution sampled at radius r converges to the 1D one (before reflections
from the square's extrapolation boundaries reach the sampled disc)."""
import numpy as np
import pytest

from classic_b200 import problems
from pyoracle import run_oracle


def _one_d(T):
    rd, solver, params, q0, _ = problems.radial_acoustics_1d(mx=1500, nout=1, tfinal=T, order=2)
    rd.clawdata.limiter = ["mc", "mc"]
    rd.clawdata.cfl_desired = 0.9
    q = run_oracle(rd, solver, params, q0, user_source="radial")[-1][2]
    return (np.arange(1500) + 0.5) * 0.001, q


def _two_d_error(n, T, r1, q1):
    rd, solver, params, _, _ = problems.radial_acoustics_2d(n=n, nout=1, tfinal=T)
    x = -1.0 + (np.arange(n) + 0.5) * 2.0 / n
    X, Y = np.meshgrid(x, x, indexing="xy")
    R = np.sqrt(X * X + Y * Y)
    q0 = np.zeros((3, n, n))
    q0[0] = problems.radial_pulse(R)
    q = run_oracle(rd, solver, params, q0)[-1][2]
    inside = R < 0.85  # the outgoing front reaches the boundary at t = 0.15
    return np.abs(q[0] - np.interp(R, r1, q1[0]))[inside].max()


def test_radial_symmetry_2d_converges_to_1d_radial_source():
    T = 0.2
    r1, q1 = _one_d(T)
    e100 = _two_d_error(100, T, r1, q1)
    e200 = _two_d_error(200, T, r1, q1)
    amp = np.abs(q1[0]).max()
    assert e200 < 0.01 * amp
    assert e200 < 0.6 * e100


def test_source_changes_the_solution_and_default_is_a_no_op():
    rd, solver, params, q0, _ = problems.radial_acoustics_1d(mx=300, nout=1, tfinal=0.3)
    with_src = run_oracle(rd, solver, params, q0, user_source="radial")[-1][2]
    default = run_oracle(rd, solver, params, q0)[-1][2]  # src1.f of src/1d: nothing
    rd.clawdata.source_split = "none"
    plain = run_oracle(rd, solver, params, q0)[-1][2]
    assert np.array_equal(default, plain)
    assert np.abs(with_src - plain).max() > 0.1


@pytest.mark.parametrize("split", ["godunov", "strang"])
def test_axisymmetric_rows_follow_the_1d_radial_run(split):
    """2D (r, z) with z-independent data: every row is the 1D radial run to
    rounding (the 2D and 1D updates group their sums differently)."""
    T = 0.2
    nr = 300
    rd, solver, params, q0, _ = problems.axisymmetric_acoustics_2d(nr=nr, nz=6, tfinal=T, nout=1,
                                                                   source_split=split, zdata=False)
    q2 = run_oracle(rd, solver, params, q0, user_source="radial")[-1][2]
    rd1, s1, p1, q1, _ = problems.radial_acoustics_1d(mx=nr, nout=1, tfinal=T, order=2,
                                                      source_split=split)
    rd1.clawdata.limiter = ["mc", "mc"]
    rd1.clawdata.cfl_desired = 0.9
    rd1.clawdata.dt_initial = 0.5
    f1 = run_oracle(rd1, s1, p1, q1, user_source="radial")[-1][2]
    for j in range(q2.shape[1]):
        assert np.abs(q2[0, j] - f1[0]).max() < 1e-11
        assert np.abs(q2[1, j] - f1[1]).max() < 1e-11
    assert np.abs(q2[2]).max() == 0.0


def test_b4step_reversing_flow_returns_the_annulus_data():
    """A before-step routine (b4step2 hook, src/2d/claw2.f:626-631) that scales
    the annulus velocities by cos(pi t / T): the data rotate forward until T/2
    and back to their start at T, apart from the scheme's diffusion and the
    per-step freezing of the velocity."""
    rd, solver, _, q0, aux = problems.advection_2d_annulus(mx=40, my=120, nout=2, tfinal=1.0)
    rd.clawdata.dt_max = 0.005
    fr = run_oracle(rd, solver, {"period": 1.0}, q0, aux, user_b4step="reversing")
    half, end = np.abs(fr[1][2] - q0).max(), np.abs(fr[2][2] - q0).max()
    assert half > 0.9 and end < 0.15
