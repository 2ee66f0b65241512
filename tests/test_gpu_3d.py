"""3D step / advance (step3 + flux3 with vc-acoustics rpn3/rpt3/rptt3) on the
GPU against the CPU oracle, through the C ABI.

The FP64 3D path rounds every multiply and add separately and adds each
cell's nine slice contributions per sweep in step3's colour order, so q, the
Courant number and the dt sequence compare bit for bit (value equality,
+0 == -0).  The piston boundary condition evaluates exp() on the device,
whose last bit may differ from the host's, so the piston example compares
to a 1e-13 tolerance and to the reference's pinned sums."""
import json
import os

import numpy as np
import pytest

from classic_b200 import problems
from classic_b200.solver import Solver, run
from helpers import frame_sum, rel_diff, same
from pyoracle import OracleGrid, run_oracle

pytestmark = pytest.mark.gpu

SIZES3 = [(7, 5, 6), (17, 9, 11), (33, 18, 15), (70, 9, 8), (8, 70, 9), (9, 8, 70), (2, 3, 4)]
BCS3 = [("extrap",) * 6,
        ("wall",) * 6,
        ("periodic",) * 6,
        ("wall", "extrap", "periodic", "periodic", "extrap", "wall"),
        ("periodic", "periodic", "wall", "extrap", "wall", "extrap")]
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "regression_sums.json")))


def _pair(rd, solver, params, q0, aux, user_bc=None):
    g = Solver(rd.clawdata, solver, params, user_bc=user_bc)
    o = OracleGrid(rd.clawdata, solver, params)
    g.set_q(q0)
    o.set_q(q0)
    g.set_aux(aux)
    o.set_aux(aux)
    return g, o


@pytest.mark.parametrize("shape", SIZES3)
@pytest.mark.parametrize("bc", BCS3)
def test_single_step_bitwise(shape, bc):
    mx, my, mz = shape
    rd, solver, params, q0, aux = problems.random_acoustics_3d(mx, my, mz, seed=mx * 7 + my * 3 + mz,
                                                               bc=bc)
    g, o = _pair(rd, solver, params, q0, aux)
    t = 0.0
    for dt in (0.004, 0.006):
        cg, co = g.step(dt), o.step(dt, t)
        t += dt
        assert cg == co
        assert same(g.get_q(), o.get_q())
    g.close()


@pytest.mark.parametrize("lim", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("order,trans", [(1, 0), (1, 10), (1, 11), (2, 0), (2, 10), (2, 11),
                                         (2, 20), (2, 21), (2, 22)])
def test_methods_bitwise(lim, order, trans):
    rd, solver, params, q0, aux = problems.random_acoustics_3d(
        21, 19, 17, seed=11, limiter=lim, order=order, trans=trans,
        bc=("wall", "extrap", "extrap", "wall", "wall", "extrap"))
    g, o = _pair(rd, solver, params, q0, aux)
    t = 0.0
    for _ in range(2):
        assert g.step(0.01) == o.step(0.01, t)
        t += 0.01
    assert same(g.get_q(), o.get_q())
    g.close()


def test_advance_dt_sequence_and_reject_path():
    """claw3's control on the device: the first dt is rejected and retried,
    then variable dt; the stats are claw3's dtv/cflv/nv."""
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(shape=(24, 20, 22),
                                                                      dt_initial=0.5)
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


def test_launches_three_sweeps_per_step():
    rd, solver, params, q0, aux = problems.random_acoustics_3d(9, 8, 7)
    g = Solver(rd.clawdata, solver, params)
    g.set_q(q0)
    g.set_aux(aux)
    n0 = g.launch_count()
    g.step(0.001)
    assert g.launch_count() - n0 == 3
    g.close()


def test_invalid_transverse_code_is_info_6():
    """src/3d/chkmth.f: method(3)=12 is not a 3D method."""
    rd, solver, params, q0, aux = problems.random_acoustics_3d(6, 6, 6, trans=12)
    g = Solver(rd.clawdata, solver, params)
    g.set_q(q0)
    g.set_aux(aux)
    info, _ = g.advance(0.0, 0.1, 0.01)
    assert info == 6
    g.close()


def test_piston_example_against_pins_and_oracle():
    """examples/acoustics_3d_heterogeneous at 20^3 (regression overrides):
    the GPU frames against the oracle's and against the reference's sums."""
    rd, solver, params, q0, aux = problems.acoustics_3d_heterogeneous()
    fg = run(rd, solver, params, q0, aux, user_bc="piston")
    fo = run_oracle(rd, solver, params, q0, aux)
    ref = GOLD["acoustics_3d_heterogeneous"]["frames"]
    for a, b in zip(fg[1:], fo[1:]):
        assert a.t == b[1]
        assert np.all(rel_diff(a.q, b[2]) <= 1e-13)
        sums = [frame_sum(a.q[m]) for m in range(3)]
        np.testing.assert_allclose(sums[0], ref[str(a.frame)][0], rtol=1e-13)
        assert np.all(np.abs(np.array(sums[1:]) - np.array(ref[str(a.frame)][1:])) < 1e-15)


def test_64_cube_advance_bitwise():
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=64)
    g, o = _pair(rd, solver, params, q0, aux)
    ig, sg = g.advance(0.0, 0.06, 0.01)
    io, so = o.advance(0.0, 0.06, 0.01)
    assert ig == io == 0 and sg["steps_taken"] == so["steps_taken"] >= 3
    assert sg["t_reached"] == so["t_reached"] and sg["dt_next"] == so["dt_next"]
    assert same(g.get_q(), o.get_q())
    g.close()


def test_full_size_256_determinism_and_mirror_symmetry():
    """At the 256^3 workload size: two runs are bitwise identical; the x -> -x
    mirror image of the data gives the mirrored solution (u odd, p v w even)
    to roundoff (the colour order of the sweeps is not mirror symmetric)."""
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=256)
    outs = []
    for qq in (q0, q0, q0[:, :, :, ::-1] * np.array([1, -1, 1, 1])[:, None, None, None]):
        g = Solver(rd.clawdata, solver, params)
        g.set_q(np.ascontiguousarray(qq))
        g.set_aux(aux)
        info, st = g.advance(0.0, 0.03, 0.01)
        assert info == 0 and st["steps_taken"] >= 3
        outs.append(g.get_q())
        g.close()
    assert same(outs[0], outs[1])
    mir = outs[2][:, :, :, ::-1] * np.array([1, -1, 1, 1])[:, None, None, None]
    assert np.all(rel_diff(mir, outs[0]) < 1e-12)


def test_fused_fp64_within_1e12_and_same_dt():
    """CLAW_FP64_FMA: the same kernels with contraction; the Courant number
    is a single product, so the dt sequence is identical."""
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=48)
    g = Solver(rd.clawdata, solver, params, precision="fp64_fma")
    o = OracleGrid(rd.clawdata, solver, params)
    for s in (g, o):
        s.set_q(q0)
        s.set_aux(aux)
    ig, sg = g.advance(0.0, 0.1, 0.01)
    io, so = o.advance(0.0, 0.1, 0.01)
    assert ig == io == 0
    for key in ("t_reached", "dt_next", "steps_taken", "cfl_max_seen"):
        assert sg[key] == so[key], key
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 1e-12)
    g.close()


def test_fp32_tracks_fp64():
    """CLAW_FP32: FP32 update, FP64 Courant number / dt / time."""
    rd, solver, params, q0, aux = problems.heterogeneous_acoustics_3d(n=48)
    g = Solver(rd.clawdata, solver, params, precision="fp32")
    o = OracleGrid(rd.clawdata, solver, params)
    for s in (g, o):
        s.set_q(q0)
        s.set_aux(aux)
    ig, sg = g.advance(0.0, 0.1, 0.01)
    io, so = o.advance(0.0, 0.1, 0.01)
    assert ig == io == 0
    assert abs(sg["t_reached"] - so["t_reached"]) < 1e-12
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= 5e-5)
    g.close()


def _fast_pair(rd, solver, params, q0, aux, precision):
    g = Solver(rd.clawdata, solver, params, precision=precision)
    o = OracleGrid(rd.clawdata, solver, params)
    for s in (g, o):
        s.set_q(q0)
        s.set_aux(aux)
    return g, o


@pytest.mark.parametrize("lim", [0, 1, 3, 4])
@pytest.mark.parametrize("order,trans", [(1, 0), (1, 11), (2, 0), (2, 10), (2, 11),
                                         (2, 20), (2, 21), (2, 22)])
@pytest.mark.parametrize("precision,tol", [("fp64_fma", 1e-12), ("fp32", 5e-5)])
def test_fast_kernel_methods(lim, order, trans, precision, tol):
    """The contracted / FP32 sweep kernel over every transverse code (codes
    without double-transverse splits take its extra pair barrier) and ragged
    tiles: the same Courant numbers (to FP32 speeds), q within the build's
    tolerance."""
    rd, solver, params, q0, aux = problems.random_acoustics_3d(
        37, 19, 23, seed=5, limiter=lim, order=order, trans=trans,
        bc=("wall", "extrap", "periodic", "periodic", "wall", "extrap"))
    g, o = _fast_pair(rd, solver, params, q0, aux, precision)
    t = 0.0
    for _ in range(3):
        cg, co = g.step(0.01), o.step(0.01, t)
        t += 0.01
        if precision == "fp64_fma":
            assert cg == co
        assert abs(cg - co) <= 1e-6 * abs(co)
    assert np.all(rel_diff(g.get_q(), o.get_q()) <= tol)
    g.close()


@pytest.mark.parametrize("shape", [(2, 3, 4), (70, 9, 8), (8, 70, 9), (9, 8, 70), (33, 18, 15)])
def test_fast_kernel_ragged_sizes(shape):
    mx, my, mz = shape
    rd, solver, params, q0, aux = problems.random_acoustics_3d(mx, my, mz, seed=mx + my + mz,
                                                               bc=("extrap",) * 6)
    for precision, tol in (("fp64_fma", 1e-12), ("fp32", 5e-5)):
        g, o = _fast_pair(rd, solver, params, q0, aux, precision)
        t = 0.0
        for dt in (0.004, 0.006):
            g.step(dt)
            o.step(dt, t)
            t += dt
        assert np.all(rel_diff(g.get_q(), o.get_q()) <= tol)
        g.close()
