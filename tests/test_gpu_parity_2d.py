"""2D step / advance on the GPU against the CPU oracle, through the C ABI.

The FP64 path is built with separately rounded multiplies and adds in the
reference's order of operations, so the comparison is bit-for-bit (value
equality, +0 == -0) for q, the Courant number and the dt sequence."""
import os
import numpy as np
import pytest

from classic_b200 import problems
from classic_b200.solver import Solver
from helpers import rel_diff, same
from pyoracle import OracleGrid

pytestmark = pytest.mark.gpu

SIZES = [(7, 5), (29, 31), (57, 100), (130, 67), (3, 64), (64, 2)]
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


@pytest.mark.parametrize("mx,my", SIZES)
@pytest.mark.parametrize("bc", BCS)
def test_single_step_bitwise(mx, my, bc):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(mx, my, seed=mx * 131 + my, bc=bc)
    g, o = _pair(rd, solver, params, q0)
    for dt in (0.004, 0.006):
        cg, co = g.step(dt), o.step(dt)
        assert cg == co
        assert same(g.get_q(), o.get_q())
    g.close()


@pytest.mark.parametrize("lim", ["none", "minmod", "superbee", "vanleer", "mc", 5])
@pytest.mark.parametrize("order,trans", [(1, 0), (1, 1), (2, 0), (2, 1), (2, 2)])
def test_methods_bitwise(lim, order, trans):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(45, 38, seed=7, limiter=lim,
                                                            order=order, trans=trans,
                                                            bc=("wall", "extrap", "extrap", "wall"))
    g, o = _pair(rd, solver, params, q0)
    for _ in range(3):
        assert g.step(0.005) == o.step(0.005)
    assert same(g.get_q(), o.get_q())
    g.close()


def test_advance_matches_dt_sequence_and_reject_path():
    """claw2 control on the device: first dt too large -> rejected and
    retried; variable dt; stats equal to claw2's dtv/cflv/nv."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=96, nout=3, tfinal=0.3,
                                                            dt_initial=0.5)
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


def test_fixed_dt_and_info_codes():
    rd, solver, params, q0, _ = problems.random_acoustics_2d(40, 40, seed=1)
    cd = rd.clawdata
    cd.dt_variable = False
    g, o = _pair(rd, solver, params, q0)
    ig, sg = g.advance(0.0, 0.02, 0.005)
    io, so = o.advance(0.0, 0.02, 0.005)
    assert ig == io == 0 and sg["steps_taken"] == so["steps_taken"] == 4
    assert same(g.get_q(), o.get_q())
    assert g.advance(0.0, 0.1, 0.03)[0] == 2
    assert g.advance(0.0, 0.4, 0.2)[0] == 12
    g.close()


def test_radial_full_run_bitwise():
    """The 2D radial acoustics workload (MC, transverse 2) to t_final = 0.6
    at 128^2: every frame bit-identical to the oracle."""
    from classic_b200.solver import run
    from pyoracle import run_oracle
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=128, nout=4, tfinal=0.6)
    fg = run(rd, solver, params, q0)
    fo = run_oracle(rd, solver, params, q0)
    assert len(fg) == len(fo)
    for a, b in zip(fg, fo):
        assert a.t == b[1]
        assert same(a.q, b[2])


def test_annulus_capacity_bitwise():
    """Capacity, aux-dependent solver, periodic y: the reference's only 2D
    regression case, bit-identical to the oracle frame by frame."""
    from classic_b200.solver import run
    from pyoracle import run_oracle
    rd, solver, params, q0, aux = problems.advection_2d_annulus()
    fg = run(rd, solver, params, q0, aux)
    fo = run_oracle(rd, solver, params, q0, aux)
    for a, b in zip(fg, fo):
        assert a.t == b[1]
        assert same(a.q, b[2])


def test_full_size_4096_step_bitwise():
    """The benchmark size (4096^2) for two steps: bit-identical to the oracle."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=4096)
    g, o = _pair(rd, solver, params, q0)
    dx = 2.0 / 4096
    for dt in (0.9 * dx / 2.0, 0.85 * dx / 2.0):
        assert g.step(dt) == o.step(dt)
    assert same(g.get_q(), o.get_q())
    g.close()


def test_determinism_and_symmetry_1024():
    """Size-independent properties at 1024^2 over 50 steps: two runs are
    bit-identical; the radially symmetric data stays mirror symmetric
    (p even, u odd in x) to roundoff."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=1024)
    runs = []
    for _ in range(2):
        g = Solver(rd.clawdata, solver, params)
        g.set_q(q0)
        for _ in range(50):
            g.step(0.9 * (2.0 / 1024) / 2.0)
        runs.append(g.get_q())
        g.close()
    assert same(runs[0], runs[1])
    q = runs[0]
    assert np.max(np.abs(q[0] - q[0][:, ::-1])) < 1e-12
    assert np.max(np.abs(q[1] + q[1][:, ::-1])) < 1e-12
    assert np.max(np.abs(q[0] - q[0].T)) < 1e-12


def test_fp32_variant_tracks_fp64():
    """FP32 update path, FP64 CFL/dt/time: within single-precision error of
    the FP64 oracle after 20 steps."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=256, nout=1, tfinal=0.05)
    g, o = _pair(rd, solver, params, q0, precision="fp32")
    ig, sg = g.advance(0.0, 0.05, 0.01)
    io, so = o.advance(0.0, 0.05, 0.01)
    assert ig == io == 0 and sg["steps_taken"] == so["steps_taken"]
    assert np.all(rel_diff(g.get_q(), o.get_q()) < 2e-5)
    g.close()


# ---------------------------------------------------------------------------
# Characteristic-variable path (CLAW_FP64_FMA): same algorithm with fused
# multiply-adds and strength ratios; same dt sequence, q within 1e-12.
@pytest.mark.parametrize("bc", BCS)
def test_fast_fp64_matches_oracle(bc):
    rd, solver, params, q0, _ = problems.random_acoustics_2d(61, 45, seed=11, bc=bc)
    g, o = _pair(rd, solver, params, q0, precision="fp64_fma")
    for _ in range(20):
        assert g.step(0.004) == o.step(0.004)  # Courant number bit-identical
    assert np.all(rel_diff(g.get_q(), o.get_q()) < 1e-12)
    g.close()


def test_fast_fp64_full_run_4096_within_1e12():
    """The benchmark workload end to end: 2D radial acoustics, 4096^2, MC,
    t = 0 -> 0.6 (~2700 steps).  The fast path against the reference-order
    path (itself bit-identical to the oracle): identical dt sequence, max
    relative difference per field <= 1e-12."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=4096)
    out = {}
    for prec in ("fp64", "fp64_fma"):
        s = Solver(rd.clawdata, solver, params, precision=prec)
        s.set_q(q0)
        info, st = s.advance(0.0, 0.6, 0.01)
        assert info == 0
        out[prec] = (s.get_q(), st)
        s.close()
    (qa, sa), (qb, sb) = out["fp64"], out["fp64_fma"]
    for key in ("t_reached", "steps_taken", "dt_next", "cfl_max_seen", "steps_rejected"):
        assert sa[key] == sb[key], key
    assert sa["steps_taken"] > 2000
    d = rel_diff(qb, qa)
    assert np.all(d <= 1e-12), d


def test_config2_1024_against_oracle_50_steps():
    """The 1024^2 size of the radial-acoustics workload, every arithmetic
    against the CPU restatement itself (not through the reference-order GPU
    kernel): claw2 from t = 0 to 0.045 (51 steps at Courant number 0.9).
    Reference order: bit-identical q and dt/Courant returns.  Fused FP64 (the
    benchmark's arithmetic): the same dt sequence and Courant numbers, max
    relative difference per field <= 1e-12.  FP32 update: the same number of
    steps, <= 1e-5."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=1024)
    o = OracleGrid(rd.clawdata, solver, params)
    o.set_q(q0)
    info_o, so = o.advance(0.0, 0.045, 0.01)
    assert info_o == 0 and so["steps_taken"] >= 50
    qo = o.get_q()
    for prec in ("fp64", "fp64_fma", "fp32"):
        s = Solver(rd.clawdata, solver, params, precision=prec)
        s.set_q(q0)
        info, st = s.advance(0.0, 0.045, 0.01)
        q = s.get_q()
        s.close()
        assert info == 0
        assert st["steps_taken"] == so["steps_taken"], prec
        if prec == "fp32":
            assert np.all(rel_diff(q, qo) <= 1e-5)
            continue
        for key in ("t_reached", "dt_next", "cfl_max_seen", "cfl_last", "dt_min", "dt_max_taken"):
            assert st[key] == so[key], (prec, key)
        if prec == "fp64":
            assert same(q, qo)
        else:
            d = rel_diff(q, qo)
            assert np.all(d <= 1e-12), d


@pytest.mark.parametrize("lim", ["minmod", "superbee", "vanleer", ("mc", "minmod"), ("vanleer", "none")])
@pytest.mark.parametrize("order,trans", [(1, 0), (1, 1), (2, 0), (2, 1), (2, 2)])
def test_fast_fp32_methods_track_fp64(order, trans, lim):
    """The FP32 characteristic kernel at every (order, transverse_waves)
    combination, each limiter compiled in or a pair read at run time, every
    BC class, against the CPU restatement."""
    for bc in BCS:
        rd, solver, params, q0, _ = problems.random_acoustics_2d(53, 41, seed=4, bc=bc, order=order,
                                                                trans=trans)
        rd.clawdata.limiter = list(lim) if isinstance(lim, tuple) else [lim, lim]
        g, o = _pair(rd, solver, params, q0, precision="fp32")
        for _ in range(10):
            cg, co = g.step(0.004), o.step(0.004)
            assert abs(cg - co) <= 1e-7 * co
        assert np.all(rel_diff(g.get_q(), o.get_q()) < 1e-5)
        g.close()


def test_fast_fp32_tracks_fp64_all_bcs():
    for bc in BCS:
        rd, solver, params, q0, _ = problems.random_acoustics_2d(70, 33, seed=2, bc=bc)
        g, o = _pair(rd, solver, params, q0, precision="fp32")
        for _ in range(10):
            cg, co = g.step(0.004), o.step(0.004)
            assert abs(cg - co) <= 1e-7 * co
        assert np.all(rel_diff(g.get_q(), o.get_q()) < 1e-5)
        g.close()


def test_frames_written_and_restart_continues(tmp_path):
    """run() with outdir writes fort.q/fort.t per frame; a restart from frame
    1 reads that file's q and t and continues frames 2.. exactly as claw2
    does from that state (checked against the oracle started from the same
    file)."""
    from classic_b200 import frames as F
    from classic_b200.solver import run
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=64, nout=3, tfinal=0.3)
    out = str(tmp_path)
    fr = run(rd, solver, params, q0, outdir=out)
    assert [f.frame for f in fr] == [0, 1, 2, 3]
    for k in range(4):
        t, q = F.read_frame(out, k)
        assert abs(t - fr[k].t) <= 1e-15 and np.allclose(q, fr[k].q, rtol=1e-15, atol=1e-99)
    info_lines = open(os.path.join(out, "fort.info")).read().split("\n")
    assert len(info_lines) == 3 * 9 + 1
    for k in range(1, 4):
        rec = info_lines[(k - 1) * 9:k * 9]
        assert rec[0] == "tend =" + F.fortran_d(fr[k].t)
        assert rec[1] == "info =    0"
        assert rec[4] == "last dt =" + F.fortran_d(fr[k].stats["dt_next"])
        assert rec[7] == "steps taken =" + F.fortran_i(fr[k].stats["steps_taken"], 4)
    rd.clawdata.restart = True
    rd.clawdata.restart_file = "fort.q0001"
    fr2 = run(rd, solver, params, None, outdir=out)
    assert [f.frame for f in fr2] == [2, 3]
    t1, q1 = F.read_frame(out, 1)
    o = OracleGrid(rd.clawdata, solver, params)
    o.set_q(q1)
    dtout = 0.3 / 3
    info, st = o.advance(t1, t1 + dtout, float(rd.clawdata.dt_initial))
    assert info == 0 and st["t_reached"] == fr2[0].t
    assert same(fr2[0].q, o.get_q())


def test_steps_max_windows_equal_one_advance():
    """nv(1) per call (claw_set_steps_max): each call stops after 7 steps with
    info 11 and dtv(5); chaining the calls as claw2ez chains frames gives the
    same state, step count and dt as one call (and the oracle's claw2 with
    the same nv(1) returns the same info)."""
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=96)
    one = Solver(rd.clawdata, solver, params)
    one.set_q(q0)
    info, st = one.advance(0.0, 0.2, 0.01)
    assert info == 0
    win = Solver(rd.clawdata, solver, params)
    win.set_q(q0)
    win.set_steps_max(7)
    t, dt, steps, calls = 0.0, 0.01, 0, 0
    while t < 0.2:
        info_w, sw = win.advance(t, 0.2, dt)
        assert info_w in (0, 11)
        assert sw["steps_taken"] <= 7
        if info_w == 11:
            assert sw["steps_taken"] == 7 and sw["t_reached"] < 0.2
        t, dt = sw["t_reached"], sw["dt_next"]
        steps += sw["steps_taken"]
        calls += 1
    assert steps == st["steps_taken"] and calls > 2
    assert dt == st["dt_next"] and t == st["t_reached"]
    assert same(win.get_q(), one.get_q())
    rd.clawdata.steps_max = 7
    o = OracleGrid(rd.clawdata, solver, params)
    o.set_q(q0)
    info_o, so = o.advance(0.0, 0.2, 0.01)
    g = Solver(rd.clawdata, solver, params)
    g.set_q(q0)
    info_g, sg = g.advance(0.0, 0.2, 0.01)
    assert info_o == info_g == 11 and sg["steps_taken"] == so["steps_taken"] == 7
    assert same(g.get_q(), o.get_q())
    for s in (one, win, g):
        s.close()
