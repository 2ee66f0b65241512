"""Dimensionally split steps (2D Godunov and Strang, src/2d/dimsp2.f +
src/2d/step2ds.f90; 3D Godunov, src/3d/dimsp3.f + src/3d/step3ds.f90) on the
GPU against the CPU oracle, through the C ABI.

The fused split kernel applies the x-, y- (and Strang's second x-) sweeps to
each row as the warp passes it, in step2ds's order of operations, so q, the
Courant number and the dt sequence compare bit for bit (value equality,
+0 == -0) with the oracle's sweep-by-sweep restatement."""
import numpy as np
import pytest

from classic_b200 import problems
from classic_b200.solver import Solver, run
from helpers import rel_diff, same
from pyoracle import OracleGrid, run_oracle

pytestmark = pytest.mark.gpu

SPLITS = ["godunov", "strang"]
SIZES = [(7, 5), (29, 31), (57, 100), (130, 67), (3, 64), (64, 2), (25, 9), (49, 13)]
BCS = [("extrap", "extrap", "extrap", "extrap"),
       ("wall", "wall", "wall", "wall"),
       ("periodic", "periodic", "periodic", "periodic"),
       ("wall", "extrap", "periodic", "periodic"),
       ("periodic", "periodic", "extrap", "wall")]


def _pair(rd, solver, params, q0, aux=None, precision="fp64"):
    g = Solver(rd.clawdata, solver, params, precision)
    o = OracleGrid(rd.clawdata, solver, params)
    g.set_q(q0)
    o.set_q(q0)
    if aux is not None:
        g.set_aux(aux)
        o.set_aux(aux)
    return g, o


@pytest.mark.parametrize("split", SPLITS)
@pytest.mark.parametrize("mx,my", SIZES)
@pytest.mark.parametrize("bc", BCS)
def test_single_step_bitwise(split, mx, my, bc):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(mx, my, seed=mx * 131 + my, bc=bc)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0)
    for dt in (0.004, 0.006):
        cg, co = g.step(dt), o.step(dt)
        assert cg == co
        assert same(g.get_q(), o.get_q())
    g.close()


@pytest.mark.parametrize("split", SPLITS)
@pytest.mark.parametrize("lim", ["none", "minmod", "superbee", "vanleer", "mc", 5])
@pytest.mark.parametrize("order", [1, 2])
def test_methods_bitwise(split, lim, order):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(45, 38, seed=7, limiter=lim,
                                                            order=order,
                                                            bc=("wall", "extrap", "extrap", "wall"))
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0)
    for _ in range(3):
        assert g.step(0.005) == o.step(0.005)
    assert same(g.get_q(), o.get_q())
    g.close()


@pytest.mark.parametrize("split", SPLITS)
def test_fwaves_bitwise(split):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(33, 40, seed=12, limiter="vanleer")
    rd.clawdata.dimensional_split = split
    rd.clawdata.use_fwaves = True
    g, o = _pair(rd, solver, params, q0)
    for _ in range(2):
        assert g.step(0.005) == o.step(0.005)
    assert same(g.get_q(), o.get_q())
    g.close()


@pytest.mark.parametrize("split", SPLITS)
def test_advance_dt_sequence_and_reject_path(split):
    """claw2 around dimsp2: the first dt is rejected on a sweep's Courant
    number and retried; variable dt; stats equal to claw2's."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=96, nout=3, tfinal=0.3,
                                                            dt_initial=0.5)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0)
    t, dt = 0.0, 0.5
    for k in range(3):
        ig, sg = g.advance(t, t + 0.1, dt)
        io, so = o.advance(t, t + 0.1, dt)
        assert ig == io == 0
        for key in ("t_reached", "dt_min", "dt_max_taken", "dt_next", "cfl_max_seen",
                    "cfl_last", "steps_taken"):
            assert sg[key] == so[key], key
        if k == 0:
            assert sg["steps_rejected"] >= 1
        assert same(g.get_q(), o.get_q())
        t, dt = sg["t_reached"], sg["dt_next"]
    g.close()


@pytest.mark.parametrize("split", SPLITS)
@pytest.mark.parametrize("shape", [(40, 20), (20, 40)])
def test_abandoned_sweep_reports_its_courant_number(split, shape):
    """A step whose x-sweep (40 x 20) or y-sweep (20 x 40) exceeds cfl_max:
    dimsp2 returns that sweep's Courant number (claw2 then discards the
    state, so only the number is compared)."""
    rd, solver, params, q0, _ = problems.random_acoustics_2d(*shape, seed=4)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0)
    # c = 2: Courant numbers 40 dt (x, 40 cells) and 20 dt; Strang's x-sweeps take dt/2
    dt = 0.03 if (split == "godunov" or shape == (20, 40)) else 0.06
    assert g.step(dt) == o.step(dt) > 1.0
    g.close()


@pytest.mark.parametrize("split", SPLITS)
def test_euler_quadrants_bitwise(split):
    rd, solver, params, q0, _ = problems.euler_quadrants(n=72, seed=3)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0)
    info_g, sg = g.advance(0.0, 0.05, 1e-3)
    info_o, so = o.advance(0.0, 0.05, 1e-3)
    assert info_g == info_o == 0
    assert sg["steps_taken"] == so["steps_taken"] and sg["dt_next"] == so["dt_next"]
    assert same(g.get_q(), o.get_q())
    g.close()


@pytest.mark.parametrize("split", SPLITS)
def test_annulus_capacity_bitwise(split):
    """Capacity + aux (examples/advection_2d_annulus) under splitting."""
    rd, solver, params, q0, aux = problems.advection_2d_annulus()
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0, aux)
    info_g, sg = g.advance(0.0, 0.1, 0.002)
    info_o, so = o.advance(0.0, 0.1, 0.002)
    assert info_g == info_o == 0
    assert sg["steps_taken"] == so["steps_taken"] and sg["cfl_max_seen"] == so["cfl_max_seen"]
    assert same(g.get_q(), o.get_q())
    g.close()


@pytest.mark.parametrize("split", SPLITS)
def test_large_grid_chunks_bitwise(split):
    """Enough rows that warps march in several row chunks per strip."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=600, dt_initial=0.0015)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0)
    for _ in range(2):  # Courant number 0.9
        assert g.step(0.0015) == o.step(0.0015)
    assert same(g.get_q(), o.get_q())
    g.close()


@pytest.mark.parametrize("split", SPLITS)
def test_fp32_tracks_fp64(split):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(70, 50, seed=8)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0, precision="fp32")
    for _ in range(3):
        cg, co = g.step(0.005), o.step(0.005)
        assert abs(cg - co) <= 1e-12
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 5e-6)
    g.close()


# ------------------------------------------------------------------- 3D ---
SIZES3 = [(7, 5, 6), (17, 9, 11), (33, 18, 15), (70, 9, 8), (8, 70, 9), (9, 8, 70), (2, 3, 4)]
BCS3 = [("extrap",) * 6,
        ("wall",) * 6,
        ("periodic",) * 6,
        ("wall", "extrap", "periodic", "periodic", "extrap", "wall"),
        ("periodic", "periodic", "wall", "extrap", "wall", "extrap")]


@pytest.mark.parametrize("shape", SIZES3)
@pytest.mark.parametrize("bc", BCS3)
def test_3d_single_step_bitwise(shape, bc):
    rd, solver, params, q0, aux = problems.random_acoustics_3d(*shape, seed=sum(shape), bc=bc)
    rd.clawdata.dimensional_split = "godunov"
    g, o = _pair(rd, solver, params, q0, aux)
    t = 0.0
    for dt in (0.004, 0.006):
        cg, co = g.step(dt), o.step(dt, t)
        t += dt
        assert cg == co
        assert same(g.get_q(), o.get_q())
    g.close()


@pytest.mark.parametrize("lim", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("order", [1, 2])
def test_3d_methods_bitwise(lim, order):
    rd, solver, params, q0, aux = problems.random_acoustics_3d(
        21, 19, 17, seed=11, limiter=lim, order=order,
        bc=("wall", "extrap", "extrap", "wall", "wall", "extrap"))
    rd.clawdata.dimensional_split = "strang"  # 3D runs Godunov for any request
    g, o = _pair(rd, solver, params, q0, aux)
    assert o.method[2] == -1
    t = 0.0
    for _ in range(2):
        assert g.step(0.01) == o.step(0.01, t)
        t += 0.01
    assert same(g.get_q(), o.get_q())
    g.close()


def test_3d_advance_and_reject_path():
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(shape=(24, 20, 22),
                                                                      dt_initial=0.5)
    rd.clawdata.dimensional_split = "godunov"
    g, o = _pair(rd, solver, params, q0, aux)
    t, dt = 0.0, 0.5
    for k in range(3):
        ig, sg = g.advance(t, t + 0.1, dt)
        io, so = o.advance(t, t + 0.1, dt)
        assert ig == io == 0
        for key in ("t_reached", "dt_min", "dt_max_taken", "dt_next", "cfl_max_seen",
                    "cfl_last", "steps_taken"):
            assert sg[key] == so[key], key
        if k == 0:
            assert sg["steps_rejected"] >= 1
        assert same(g.get_q(), o.get_q())
        t, dt = sg["t_reached"], sg["dt_next"]
    g.close()


def test_3d_piston_example_split():
    """examples/acoustics_3d_heterogeneous at 20^3 with dimensional splitting:
    the piston's exp() on the device may differ in the last bit."""
    rd, solver, params, q0, aux = problems.acoustics_3d_heterogeneous()
    rd.clawdata.dimensional_split = "godunov"
    fg = run(rd, solver, params, q0, aux, user_bc="piston")
    fo = run_oracle(rd, solver, params, q0, aux)
    for a, b in zip(fg[1:], fo[1:]):
        assert a.t == b[1]
        assert np.all(rel_diff(a.q, b[2]) <= 1e-13)


def test_3d_64_cube_advance_bitwise():
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=64)
    rd.clawdata.dimensional_split = "godunov"
    g, o = _pair(rd, solver, params, q0, aux)
    ig, sg = g.advance(0.0, 0.06, 0.01)
    io, so = o.advance(0.0, 0.06, 0.01)
    assert ig == io == 0 and sg["steps_taken"] == so["steps_taken"] >= 3
    assert sg["dt_next"] == so["dt_next"]
    assert same(g.get_q(), o.get_q())
    g.close()


def test_3d_fp32_tracks_fp64():
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=40)
    rd.clawdata.dimensional_split = "godunov"
    g, o = _pair(rd, solver, params, q0, aux, precision="fp32")
    ig, sg = g.advance(0.0, 0.1, 0.01)
    io, so = o.advance(0.0, 0.1, 0.01)
    assert ig == io == 0
    assert abs(sg["t_reached"] - so["t_reached"]) < 1e-12
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 5e-5)
    g.close()


@pytest.mark.parametrize("split", SPLITS)
def test_fused_fp64_within_1e12(split):
    """CLAW_FP64_FMA: the split kernels built with contraction."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=200, nout=1, tfinal=0.05)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0, precision="fp64_fma")
    ig, sg = g.advance(0.0, 0.05, 0.004)
    io, so = o.advance(0.0, 0.05, 0.004)
    assert ig == io == 0
    for key in ("t_reached", "dt_next", "steps_taken", "cfl_max_seen"):
        assert sg[key] == so[key], key
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-12)
    g.close()


# Characteristic-variable split kernel (constant-coefficient acoustics in the
# contracted FP64 and FP32 builds, char2ds.cuh): the same dimsp2 sweeps, q
# within 1e-12 of the oracle, Courant numbers and dt sequence identical.
@pytest.mark.parametrize("split", SPLITS)
@pytest.mark.parametrize("mx,my", SIZES + [(121, 47), (300, 9)])
@pytest.mark.parametrize("bc", BCS)
def test_char_split_steps_within_1e12(split, mx, my, bc):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(mx, my, seed=3 * mx + my, bc=bc)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0, precision="fp64_fma")
    # Courant numbers 0.8 and 0.9 (c = 2 on [-1, 1]^2): a sweep above cfl_max
    # would end dimsp2's step early, which claw2 then rejects
    for frac in (0.8, 0.9):
        dt = frac / max(mx, my)
        cg, co = g.step(dt), o.step(dt)
        assert cg == co
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-12)
    g.close()


@pytest.mark.parametrize("split", SPLITS)
@pytest.mark.parametrize("lim", ["none", "minmod", "superbee", "vanleer", "mc", ("mc", "vanleer"), ("minmod", 5)])
def test_char_split_limiters_within_1e12(split, lim):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(130, 67, seed=11,
                                                            bc=("wall", "extrap", "periodic", "periodic"))
    rd.clawdata.dimensional_split = split
    rd.clawdata.limiter = list(lim) if isinstance(lim, tuple) else [lim, lim]
    g, o = _pair(rd, solver, params, q0, precision="fp64_fma")
    for _ in range(4):
        assert g.step(0.005) == o.step(0.005)
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-12)
    g.close()


@pytest.mark.parametrize("split", SPLITS)
def test_char_split_advance_reject_and_abandon(split):
    """claw2 with dimsp2 on the characteristic split kernel: a first dt far too
    large (an abandoned sweep, then retries), then variable dt over three
    frames; every statistic equal to the oracle's."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=96, dt_initial=0.5)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0, precision="fp64_fma")
    t, dg, do = 0.0, 0.5, 0.5
    for _ in range(3):
        ig, sg = g.advance(t, t + 0.1, dg)
        io, so = o.advance(t, t + 0.1, do)
        assert ig == io == 0
        for key in ("t_reached", "dt_min", "dt_max_taken", "dt_next", "cfl_max_seen", "cfl_last",
                    "steps_taken"):
            assert sg[key] == so[key], key
        assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-12)
        t, dg, do = sg["t_reached"], sg["dt_next"], so["dt_next"]
    g.close()


@pytest.mark.parametrize("split", SPLITS)
@pytest.mark.parametrize("bc", BCS)
def test_char_split_fp32_all_bcs(split, bc):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(90, 41, seed=5, bc=bc)
    rd.clawdata.dimensional_split = split
    g, o = _pair(rd, solver, params, q0, precision="fp32")
    for _ in range(3):
        cg, co = g.step(0.005), o.step(0.005)
        assert abs(cg - co) <= 1e-12
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 5e-6)
    g.close()


def test_3d_fused_fp64_within_1e12():
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=40)
    rd.clawdata.dimensional_split = "godunov"
    g, o = _pair(rd, solver, params, q0, aux, precision="fp64_fma")
    ig, sg = g.advance(0.0, 0.1, 0.01)
    io, so = o.advance(0.0, 0.1, 0.01)
    assert ig == io == 0
    for key in ("t_reached", "dt_next", "steps_taken"):
        assert sg[key] == so[key], key
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-12)
    g.close()
