"""Dimensional splitting in the CPU oracle (src/2d/dimsp2.f + step2ds.f90,
src/3d/dimsp3.f + step3ds.f90).

The reference ships no regression data for the split methods, so the
restatement is checked through exact identities it must satisfy:
  * data that vary along x only make every y-wave (and z-wave) zero, so a
    Godunov-split step equals an unsplit step without transverse propagation
    bit for bit; for data that vary along y only the two differ in rounding
    alone (step2 adds the y increments as qnew + (qadd - dtdy*df - dtdx*dg),
    src/2d/step2.f90:222-226, step2ds as (qnew + qadd) - dtdy*df,
    src/2d/step2ds.f90:252-254);
  * Strang splitting's two x half-sweeps equal two unsplit half steps away
    from the x boundaries (the second half-sweep reuses the ghost cells of the
    first; src/2d/dimsp2.f:88-90);
  * with periodic boundaries Godunov splitting conserves every field to
    roundoff (Strang's last x half-sweep reads ghost columns that were never
    x-updated, so it does not, exactly as in the reference)."""
import numpy as np
import pytest

from classic_b200 import problems
from pyoracle import OracleGrid

pytestmark = pytest.mark.filterwarnings("ignore")


def _grid(rd, solver, params, q0, aux=None):
    g = OracleGrid(rd.clawdata, solver, params)
    g.set_q(q0)
    if aux is not None:
        g.set_aux(aux)
    return g


def _x_only(q0):
    return np.ascontiguousarray(np.broadcast_to(q0[:, :1, :], q0.shape))


def _y_only(q0):
    return np.ascontiguousarray(np.broadcast_to(q0[:, :, :1], q0.shape))


@pytest.mark.parametrize("limiter", ["minmod", "superbee", "vanleer", "mc"])
@pytest.mark.parametrize("shape", [(_x_only, 1), (_y_only, 2)])
def test_godunov_on_one_dimensional_data_equals_unsplit(limiter, shape):
    make, axis = shape
    rd, solver, params, q0, _ = problems.random_acoustics_2d(37, 29, seed=3, limiter=limiter,
                                                             bc=("wall", "extrap", "periodic",
                                                                 "periodic") if axis == 1 else
                                                             ("periodic", "periodic", "wall",
                                                              "extrap"))
    q0 = make(q0)
    if axis == 1:
        q0[2] = 0.0  # v = 0: nothing moves along y
    else:
        q0[1] = 0.0
    cd = rd.clawdata
    cd.transverse_waves = 0
    ref = _grid(rd, solver, params, q0)
    cd.dimensional_split = "godunov"
    spl = _grid(rd, solver, params, q0)
    assert spl.method[2] == -1
    for dt in (0.02, 0.024, 0.022):  # Courant numbers below 1 in both directions
        c_ref, c_spl = ref.step(dt), spl.step(dt)
        a, b = ref.get_q(), spl.get_q()
        if axis == 1:
            assert c_ref == c_spl
            assert np.array_equal(a, b)
        else:
            assert abs(c_ref - c_spl) <= 1e-15
            assert np.all(np.abs(a - b) <= 1e-14 * (np.abs(a) + 1e-300))


def test_strang_equals_two_half_steps_away_from_the_x_boundaries():
    rd, solver, params, q0, _ = problems.random_acoustics_2d(41, 7, seed=5, limiter="mc")
    q0 = _x_only(q0)
    q0[2] = 0.0
    cd = rd.clawdata
    cd.transverse_waves = 0
    ref = _grid(rd, solver, params, q0)
    cd.dimensional_split = "strang"
    spl = _grid(rd, solver, params, q0)
    assert spl.method[2] == -2
    dt = 0.04
    c1 = ref.step(dt / 2)
    c2 = ref.step(dt / 2)
    c = spl.step(dt)
    assert c == max(c1, c2) or abs(c - max(c1, c2)) < 1e-15
    a, b = ref.get_q(), spl.get_q()
    assert np.array_equal(a[:, :, 2:-2], b[:, :, 2:-2])


@pytest.mark.parametrize("solver_case", ["acoustics", "euler"])
def test_periodic_godunov_split_conserves(solver_case):
    if solver_case == "acoustics":
        rd, solver, params, q0, _ = problems.random_acoustics_2d(
            33, 27, seed=9, bc=("periodic",) * 4)
    else:
        rd, solver, params, q0, _ = problems.euler_quadrants(n=32, seed=4, bc=("periodic",) * 4)
    cd = rd.clawdata
    cd.dimensional_split = "godunov"
    g = _grid(rd, solver, params, q0)
    s0 = g.get_q().sum(axis=(1, 2))
    for _ in range(4):
        g.step(0.2 * min(2.0 / q0.shape[2], 2.0 / q0.shape[1]) if solver_case == "acoustics"
               else 2e-3)
    s1 = g.get_q().sum(axis=(1, 2))
    scale = np.abs(g.get_q()).sum(axis=(1, 2)) + 1.0
    assert np.all(np.abs(s1 - s0) <= 1e-13 * scale)


def test_split_advance_runs_claw2_control():
    """The reject / retry path of claw2 around dimsp2: a too-large first dt is
    rejected on the x-sweep's Courant number and retried."""
    rd, solver, params, q0, _ = problems.random_acoustics_2d(24, 20, seed=2)
    rd.clawdata.dimensional_split = "strang"
    g = _grid(rd, solver, params, q0)
    info, st = g.advance(0.0, 0.2, 0.5)
    assert info == 0 and st["t_reached"] == 0.2 and st["cfl_max_seen"] <= 1.0


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_3d_godunov_on_one_dimensional_data_equals_unsplit(axis):
    rd, solver, params, q0, aux = problems.random_acoustics_3d(
        13, 11, 9, seed=7, trans=0, bc=("extrap", "wall", "periodic", "periodic", "extrap", "extrap"))
    # q: [meqn][mz][my][mx]; keep the variation along one axis only
    sl = [slice(None)] + [slice(0, 1)] * 3
    sl[3 - axis] = slice(None)
    q0 = np.ascontiguousarray(np.broadcast_to(q0[tuple(sl)], q0.shape))
    for m in range(1, 4):
        if m - 1 != axis:
            q0[m] = 0.0
    # a homogeneous medium keeps the transverse jumps zero
    aux = np.ascontiguousarray(np.broadcast_to(aux[:, :1, :1, :1], aux.shape))
    cd = rd.clawdata
    ref = _grid(rd, solver, params, q0, aux)
    cd.dimensional_split = "godunov"
    spl = _grid(rd, solver, params, q0, aux)
    assert spl.method[2] == -1
    t = 0.0
    for dt in (0.02, 0.03):
        assert ref.step(dt, t) == spl.step(dt, t)
        t += dt
        assert np.array_equal(ref.get_q(), spl.get_q())
