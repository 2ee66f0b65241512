"""Known-answer properties of the oracle's 2D Euler Roe solver (no reference
pin exists for 2D Euler): the Roe property sum_k s_k W_k = f(q_R) - f(q_L)
makes the wave-propagation update conservative, so with periodic boundaries
the totals of all four conserved fields stay fixed to roundoff; and a
one-dimensional shock tube stays one-dimensional."""
import numpy as np

from classic_b200 import problems
from pyoracle import OracleGrid


def test_periodic_conservation():
    for seed in (1, 2, 3):
        rd, solver, params, q0, _ = problems.euler_quadrants(n=40, seed=seed,
                                                             bc=("periodic",) * 4)
        o = OracleGrid(rd.clawdata, solver, params)
        o.set_q(q0)
        for _ in range(10):
            o.step(0.002)
        q = o.get_q()
        scale = np.abs(q0).reshape(4, -1).sum(1)
        assert np.all(np.abs(q.reshape(4, -1).sum(1) - q0.reshape(4, -1).sum(1)) <= 1e-14 * scale)


def test_shock_tube_stays_one_dimensional():
    """Sod data varying in x only: the rows of the solution agree and the
    transverse momentum stays zero, both to roundoff (the transverse
    splitting moves y-momentum between rows that cancels only to rounding)."""
    rd, solver, params, _, _ = problems.euler_quadrants(shape=(64, 8))
    g = 1.4
    x = (np.arange(64) + 0.5) / 64
    rho = np.where(x < 0.5, 1.0, 0.125)
    p = np.where(x < 0.5, 1.0, 0.1)
    q0 = np.zeros((4, 8, 64))
    q0[0] = rho
    q0[3] = p / (g - 1.0)
    o = OracleGrid(rd.clawdata, solver, params)
    o.set_q(q0)
    info, st = o.advance(0.0, 0.15, 1e-3)
    assert info == 0
    q = o.get_q()
    assert np.max(np.abs(q[2])) < 1e-13
    assert np.max(np.abs(q - q[:, :1, :])) < 1e-13
    # the shock has moved right of the diaphragm, the rarefaction left of it
    assert q[0, 0, 40] < 0.6 and q[0, 0, 20] > 0.5
