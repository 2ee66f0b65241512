"""The 1D advection (rp1_advection) and 1D Euler (rp1_euler_with_efix)
solvers of examples/advection_1d_example1 and examples/euler_1d_wcblast in
the CPU oracle.  The reference holds no regression data for either example,
so the pins are known answers:

* advection at Courant number exactly 1 is an exact shift by one cell per
  step, at first and at second order (the correction term carries the factor
  1 - |nu|, src/1d/step1.f:150-170);
* periodic advection and walled Euler conserve mass (and Euler its energy);
* a y-invariant 2D Euler run with v = 0 (the already pinned 2D Roe solver,
  periodic in y) reproduces the 1D Euler run in every row."""
import numpy as np
import pytest

from classic_b200 import problems
from pyoracle import run_oracle


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("u", [1.0, -1.0])
def test_advection_courant_one_is_an_exact_shift(order, u):
    mx, nsteps = 200, 37
    rd, solver, params, q0, _ = problems.advection_1d_example1(mx=mx, nout=1)
    params = {"u": u}
    cd = rd.clawdata
    cd.order = order
    cd.dt_variable = False
    cd.dt_initial = 1.0 / mx
    cd.tfinal = nsteps / mx
    q = run_oracle(rd, solver, params, q0)[-1][2]
    shift = nsteps if u > 0 else -nsteps
    np.testing.assert_allclose(q, np.roll(q0, shift, axis=1), rtol=0, atol=1e-13)


def test_advection_example_conserves_and_stays_bounded():
    rd, solver, params, q0, _ = problems.advection_1d_example1(nout=4)
    frames = run_oracle(rd, solver, params, q0)
    assert len(frames) == 5 and frames[-1][1] == pytest.approx(4.0)
    for _, t, q, _ in frames:
        assert abs(q.sum() - q0.sum()) < 1e-11
        # TVD (MC limiter): no new extrema
        assert q.min() >= q0.min() - 1e-12 and q.max() <= q0.max() + 1e-12


def test_wcblast_conserves_mass_and_energy():
    rd, solver, params, q0, _ = problems.euler_1d_wcblast(mx=600, nout=2)
    frames = run_oracle(rd, solver, params, q0)
    assert frames[-1][1] == pytest.approx(0.038)
    for _, _, q, _ in frames:
        assert np.isfinite(q).all()
        assert abs(q[0].sum() - q0[0].sum()) <= 1e-12 * q0[0].sum()
        assert abs(q[2].sum() - q0[2].sum()) <= 1e-12 * q0[2].sum()
        rho = q[0]
        p = 0.4 * (q[2] - 0.5 * q[1] ** 2 / rho)
        assert rho.min() > 0 and p.min() > 0


def test_euler_1d_matches_y_invariant_2d_rows():
    mx, my, gamma = 160, 4, 1.4
    rd1, s1, p1, _, _ = problems.euler_1d_wcblast(mx=mx, nout=1, tfinal=0.01)
    x = (np.arange(mx) + 0.5) / mx
    rho = np.where(x < 0.5, 1.0, 0.125)
    pr = np.where(x < 0.5, 1.0, 0.1)
    u = np.where(x < 0.5, 0.3, -0.2)
    q1 = np.stack([rho, rho * u, pr / (gamma - 1) + 0.5 * rho * u * u])
    for cd in (rd1.clawdata,):
        cd.dt_variable, cd.dt_initial, cd.tfinal = False, 0.002, 0.06
        cd.bc_lower[0], cd.bc_upper[0] = "wall", "extrap"
    out1 = run_oracle(rd1, s1, p1, q1)[-1][2]

    rd2, s2, p2, _, _ = problems.euler_quadrants(shape=(mx, my), nout=1)
    cd = rd2.clawdata
    cd.dt_variable, cd.dt_initial, cd.tfinal = False, 0.002, 0.06
    cd.bc_lower, cd.bc_upper = ["wall", "periodic"], ["extrap", "periodic"]
    q2 = np.zeros((4, my, mx))
    q2[0], q2[1], q2[3] = q1[0], q1[1], q1[2]
    out2 = run_oracle(rd2, s2, p2, q2)[-1][2]
    assert np.abs(out2[2]).max() < 1e-13
    for j in range(my):
        for m1, m2 in ((0, 0), (1, 1), (2, 3)):
            np.testing.assert_allclose(out2[m2, j], out1[m1], rtol=1e-12, atol=1e-13)


def test_frames_are_snapshots():
    """Each frame holds its own array (one field included): advection moves
    the profile between outputs."""
    rd, solver, params, q0, _ = problems.advection_1d_example1(nout=4, tfinal=0.4)
    frames = run_oracle(rd, solver, params, q0)
    for a, b in zip(frames, frames[1:]):
        assert np.abs(a[2] - b[2]).max() > 0.1
    assert not np.shares_memory(frames[1][2], frames[2][2])
