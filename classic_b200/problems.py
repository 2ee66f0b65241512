"""Problem setups: the reference examples that carry regression pins, and the
synthetic workloads (seeded or analytic initial data of the stated shapes).

Each builder returns ``(rundata, solver, params, q0, aux)`` with q0 in the
SoA interior layout [meqn][my][mx] and aux (or None) as [maux][my+4][mx+4].
Cell centres follow the reference's qinit: x_i = xlower + (i - 0.5)*dx for
1-based i.
"""
from __future__ import annotations

import numpy as np

from .data import ClawRunData


def _centres(lower, upper, n, ghost=0):
    dx = (upper - lower) / float(np.float32(n))
    i = np.arange(1 - ghost, n + ghost + 1, dtype=np.float64)
    return lower + (i - 0.5) * dx, dx


# ------------------------------------------------------------------- 1D ---
def acoustics_1d_example1(mx=400, beta=200.0, nout=2, tfinal=1.0, output_t0=False):
    """examples/acoustics_1d_example1 (setrun.py, qinit.f90, setprob.f90) with
    the regression test's overrides (test_acoustics_1d_example1.py:17-19)."""
    rd = ClawRunData("classic", 1)
    pd = rd.new_UserData("probdata", "setprob.data")
    pd.add_param("rho", 1.0)
    pd.add_param("K", 4.0)
    pd.add_param("beta", beta)
    cd = rd.clawdata
    cd.lower[0], cd.upper[0], cd.num_cells[0] = -1.0, 1.0, mx
    cd.num_eqn, cd.num_aux, cd.capa_index = 2, 0, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = output_t0
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, 0.1, 1e99
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 500
    cd.order, cd.num_waves, cd.limiter = 2, 2, ["mc", "mc"]
    cd.bc_lower[0], cd.bc_upper[0] = "extrap", "extrap"
    x, _ = _centres(-1.0, 1.0, mx)
    q0 = np.zeros((2, mx))
    q0[0] = np.exp(-beta * (x - 0.3) ** 2)
    return rd, "acoustics_1d", {"rho": 1.0, "bulk": 4.0}, q0, None


def acoustics_1d_config(mx=800, nout=10, tfinal=1.0):
    """1D linear acoustics workload: rho=1, K=4, [-1,1], p0=exp(-100(x-0.3)^2),
    u0=0, order 2, MC, cfl 0.9, wall left / extrapolation right, 10 outputs
    to t=1 (dt_initial 0.1 as in the reference example)."""
    rd, solver, params, _, _ = acoustics_1d_example1(mx=mx, beta=100.0, nout=nout, tfinal=tfinal)
    rd.clawdata.bc_lower[0] = "wall"
    rd.clawdata.output_t0 = True
    x, _ = _centres(-1.0, 1.0, mx)
    q0 = np.zeros((2, mx))
    q0[0] = np.exp(-100.0 * (x - 0.3) ** 2)
    rd.clawdata.steps_max = 5000
    return rd, solver, params, q0, None


def advection_1d_example1(mx=200, nout=20, tfinal=4.0):
    """examples/advection_1d_example1 (setrun.py, qinit.f90, setprob.f90):
    q_t + u q_x = 0 with u = 1 on [0, 1], periodic, 200 cells, MC, cfl 0.9,
    q0 = exp(-beta (x - 0.75)^2) (beta = 400) plus 1 on 0.1 < x < 0.4; 20
    outputs to t = 4 (four periods)."""
    rd = ClawRunData("classic", 1)
    pd = rd.new_UserData("probdata", "setprob.data")
    pd.add_param("u", 1.0)
    pd.add_param("beta", 400.0)
    cd = rd.clawdata
    cd.lower[0], cd.upper[0], cd.num_cells[0] = 0.0, 1.0, mx
    cd.num_eqn, cd.num_aux, cd.capa_index = 1, 0, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = True
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, 0.1, 1e99
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 500
    cd.order, cd.num_waves, cd.limiter = 2, 1, ["mc"]
    cd.bc_lower[0], cd.bc_upper[0] = "periodic", "periodic"
    x, _ = _centres(0.0, 1.0, mx)
    q0 = np.zeros((1, mx))
    q0[0] = np.exp(-400.0 * (x - 0.75) ** 2) + np.where((x > 0.1) & (x < 0.4), 1.0, 0.0)
    return rd, "advection_1d", {"u": 1.0}, q0, None


def euler_1d_wcblast(mx=2000, nout=20, tfinal=0.038, gamma=1.4):
    """examples/euler_1d_wcblast (setrun.py, qinit.f90, setprob.f90): the
    Woodward-Colella blast waves on 2000 cells, rho = 1, u = 0,
    p = 1000 / 0.01 / 100 on x < 0.1 / 0.1..0.9 / x > 0.9, solid walls, MC on
    3 waves, cfl 0.9, dt_initial 1e-6, 20 outputs to t = 0.038."""
    rd = ClawRunData("classic", 1)
    pd = rd.new_UserData("probdata", "setprob.data")
    pd.add_param("gamma", gamma)
    cd = rd.clawdata
    cd.lower[0], cd.upper[0], cd.num_cells[0] = 0.0, 1.0, mx
    cd.num_eqn, cd.num_aux, cd.capa_index = 3, 0, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = True
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, 1e-6, 1e99
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 5000
    cd.order, cd.num_waves, cd.limiter = 2, 3, ["mc"] * 3
    cd.bc_lower[0], cd.bc_upper[0] = "wall", "wall"
    x, _ = _centres(0.0, 1.0, mx)
    g1 = gamma - 1.0
    q0 = np.zeros((3, mx))
    q0[0] = 1.0
    q0[2] = np.where(x < 0.1, 1e3 / g1, np.where(x < 0.9, 1e-2 / g1, 1e2 / g1))
    return rd, "euler_roe_1d", {"gamma": gamma}, q0, None


def radial_pulse(r, width=0.2):
    """qinit of examples/acoustics_2d_radial (qinit.f:17-28) and of its 1drad
    companion (1drad/qinit.f): p = 1 + cos(pi (r-0.5)/width) for
    |r-0.5| <= width, else 0."""
    return np.where(np.abs(r - 0.5) <= width, 1.0 + np.cos(np.pi * (r - 0.5) / width), 0.0)


def radial_acoustics_1d(mx=2000, nout=20, tfinal=1.0, order=1, source_split="godunov"):
    """examples/acoustics_2d_radial/1drad (setrun.py, qinit.f, setprob.f,
    src1.f): 1D acoustics in the radius r on [0, 1.5], rho=1, bulk=4, ndim=2
    (cylindrical symmetry) through the geometric source term of src1.f with
    Godunov source splitting; wall at r=0, extrapolation at 1.5; order 1,
    cfl 1.0, dt_initial 0.5, 20 outputs to t=1.  Run it with
    user_source="radial"."""
    rd = ClawRunData("classic", 1)
    pd = rd.new_UserData("probdata", "setprob.data")
    pd.add_param("ndim", 2)
    pd.add_param("rho", 1.0)
    pd.add_param("bulk", 4.0)
    cd = rd.clawdata
    cd.lower[0], cd.upper[0], cd.num_cells[0] = 0.0, 1.5, mx
    cd.num_eqn, cd.num_aux, cd.capa_index = 2, 0, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = True
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, 0.5, 1e99
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 1.0, 1.0, 50000
    cd.order, cd.num_waves, cd.limiter = order, 2, ["superbee", "superbee"]
    cd.source_split = source_split
    cd.bc_lower[0], cd.bc_upper[0] = "wall", "extrap"
    x, _ = _centres(0.0, 1.5, mx)
    q0 = np.zeros((2, mx))
    q0[0] = radial_pulse(x)
    return rd, "acoustics_1d", {"rho": 1.0, "bulk": 4.0, "ndim": 2}, q0, None


def axisymmetric_acoustics_2d(nr=300, nz=40, tfinal=0.4, nout=2, source_split="godunov",
                              split="unsplit", zdata=True, seed=0):
    """2D acoustics in the (r, z) half-plane [0, 1.5] x [-0.2, 0.2] of a
    cylindrically symmetric field: the radial source of
    examples/acoustics_2d_radial/1drad/src1.f on every row (run with
    user_source="radial"); wall at r=0, extrapolation at r=1.5, periodic in z.
    The 1drad pulse in r; with zdata a seeded z-dependent perturbation is
    added, otherwise every row follows the 1D radial solution."""
    rd = ClawRunData("classic", 2)
    pd = rd.new_UserData("probdata", "setprob.data")
    pd.add_param("ndim", 2)
    pd.add_param("rho", 1.0)
    pd.add_param("bulk", 4.0)
    cd = rd.clawdata
    cd.lower, cd.upper, cd.num_cells = [0.0, -0.2], [1.5, 0.2], [nr, nz]
    cd.num_eqn, cd.num_aux, cd.capa_index = 3, 0, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = True
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, 0.5, 1e99
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 50000
    cd.order, cd.transverse_waves, cd.dimensional_split = 2, 2, split
    cd.num_waves, cd.limiter = 2, ["mc", "mc"]
    cd.source_split = source_split
    cd.bc_lower, cd.bc_upper = ["wall", "periodic"], ["extrap", "periodic"]
    r, _ = _centres(0.0, 1.5, nr)
    z, _ = _centres(-0.2, 0.2, nz)
    R, Z = np.meshgrid(r, z, indexing="xy")
    q0 = np.zeros((3, nz, nr))
    q0[0] = radial_pulse(R)
    if zdata:
        rng = np.random.default_rng(seed)
        q0[0] += 0.05 * np.cos(2 * np.pi * Z / 0.4) * np.exp(-20 * (R - 0.8) ** 2)
        q0[2] = 0.01 * rng.standard_normal((nz, nr))
    return rd, "acoustics_2d", {"rho": 1.0, "bulk": 4.0, "ndim": 2}, q0, None


def acoustics_1d_heterogeneous(mx=500, nout=2, tfinal=5.0, ic=1, beta=5.0):
    """examples/acoustics_1d_heterogeneous (setrun.py, qinit.f, setaux.f,
    setprob.f) with the test's overrides (test_acoustics_1d_heterogeneous.py:23-25)."""
    rd = ClawRunData("classic", 1)
    cd = rd.clawdata
    cd.lower[0], cd.upper[0], cd.num_cells[0] = -5.0, 5.0, mx
    cd.num_eqn, cd.num_aux, cd.capa_index = 2, 2, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = False
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, 1.0, 1e9
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 50000
    cd.order, cd.num_waves, cd.limiter = 2, 2, [4, 4]
    cd.bc_lower[0], cd.bc_upper[0] = "extrap", "extrap"
    rhol, cl, rhor, cr = 1.0, 1.0, 4.0, 0.5
    zl, zr = rhol * cl, rhor * cr
    x, _ = _centres(-5.0, 5.0, mx)
    q0 = np.zeros((2, mx))
    if ic == 1:
        inside = (x > -4.0) & (x < -2.0)
        q0[0] = np.where(inside, np.sqrt(np.where(inside, 1.0 - (x + 3.0) ** 2, 0.0)), 0.0)
    elif ic == 2:
        q0[0] = np.where(x < -2.0, 1.0, 0.0)
    else:
        g = np.exp(-beta * (x + 2.0) ** 2)
        g[np.abs(g) < 1e-30] = 0.0
        q0[0] = g + np.where((x > -4.0) & (x < -3.0), 0.5, 0.0)
    q0[1] = q0[0]
    xg, _ = _centres(-5.0, 5.0, mx, ghost=2)
    aux = np.zeros((2, mx + 4))
    aux[0] = np.where(xg < 0.0, zl, zr)
    aux[1] = np.where(xg < 0.0, cl, cr)
    return rd, "vc_acoustics_1d", {}, q0, aux


# ------------------------------------------------------------------- 2D ---
def radial_acoustics_2d(n=1024, nout=20, tfinal=0.6, limiter="mc", dt_initial=0.01):
    """2D radial acoustics workload: rho=1, K=4 on [-1,1]^2 with n^2 cells;
    p0 = 1 + cos(pi (r-0.5)/0.1) for |r-0.5| < 0.1 else 1, u=v=0; order 2,
    transverse_waves 2, MC limiter, cfl 0.9, extrapolation BCs, t_final 0.6.
    (examples/acoustics_2d_radial is the same solver with a narrower pulse.)"""
    rd = ClawRunData("classic", 2)
    pd = rd.new_UserData("probdata", "setprob.data")
    pd.add_param("rho", 1.0)
    pd.add_param("bulk", 4.0)
    cd = rd.clawdata
    cd.lower, cd.upper, cd.num_cells = [-1.0, -1.0], [1.0, 1.0], [n, n]
    cd.num_eqn, cd.num_aux, cd.capa_index = 3, 0, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = True
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, dt_initial, 1e99
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 50000
    cd.order, cd.transverse_waves, cd.dimensional_split = 2, 2, "unsplit"
    cd.num_waves, cd.limiter = 2, [limiter, limiter]
    cd.bc_lower, cd.bc_upper = ["extrap", "extrap"], ["extrap", "extrap"]
    x, _ = _centres(-1.0, 1.0, n)
    X, Y = np.meshgrid(x, x, indexing="xy")  # [j][i]
    r = np.sqrt(X * X + Y * Y)
    q0 = np.zeros((3, n, n))
    q0[0] = np.where(np.abs(r - 0.5) < 0.1, 1.0 + np.cos(np.pi * (r - 0.5) / 0.1), 1.0)
    return rd, "acoustics_2d", {"rho": 1.0, "bulk": 4.0}, q0, None


def advection_2d_annulus(mx=40, my=120, nout=2, tfinal=0.5):
    """examples/advection_2d_annulus (setrun.py, qinit.f, setaux.f, mapc2p.f,
    stream.f) with the test's overrides (test_advection_2d_annulus.py:16-17):
    polar grid r in [0.2,1], theta in [0,2pi], capacity = cell area / (dr dtheta),
    edge velocities from differences of the stream function pi*(x^2+y^2)."""
    rd = ClawRunData("classic", 2)
    cd = rd.clawdata
    cd.lower, cd.upper, cd.num_cells = [0.2, 0.0], [1.0, 2.0 * np.pi], [mx, my]
    cd.num_eqn, cd.num_aux, cd.capa_index = 1, 3, 3
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = True
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, 0.1, 1e9
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 50000
    cd.order, cd.transverse_waves, cd.dimensional_split = 2, "all", "unsplit"
    cd.num_waves, cd.limiter = 1, ["vanleer"]
    cd.bc_lower, cd.bc_upper = ["extrap", "periodic"], ["extrap", "periodic"]
    xlo, ylo = 0.2, 0.0
    dxc = (1.0 - 0.2) / float(np.float32(mx))
    dyc = (2.0 * np.pi - 0.0) / float(np.float32(my))

    def mapc2p(xc, yc):
        return xc * np.cos(yc), xc * np.sin(yc)

    def stream(x, y):
        return 3.1415926535897931 * (x ** 2 + y ** 2)

    ig = np.arange(-1, mx + 3, dtype=np.float64)  # 1-based i = -1 .. mx+2
    jg = np.arange(-1, my + 3, dtype=np.float64)
    XC1 = xlo + (ig[None, :] - 1.0) * dxc
    YC1 = ylo + (jg[:, None] - 1.0) * dyc
    XC1, YC1 = np.broadcast_arrays(XC1, YC1)
    xp1, yp1 = mapc2p(XC1, YC1)
    xp2, yp2 = mapc2p(XC1, YC1 + dyc)
    xp3, yp3 = mapc2p(XC1 + dxc, YC1 + dyc)
    xp4, yp4 = mapc2p(XC1 + dxc, YC1)
    aux = np.zeros((3, my + 4, mx + 4))
    aux[0] = (stream(xp2, yp2) - stream(xp1, yp1)) / dyc
    aux[1] = -(stream(xp4, yp4) - stream(xp1, yp1)) / dxc
    xs = [xp1, xp2, xp3, xp4, xp1]
    ys = [yp1, yp2, yp3, yp4, yp1]
    area = np.zeros_like(xp1)
    for k in range(4):
        area = area + 0.5 * (ys[k] + ys[k + 1]) * (xs[k + 1] - xs[k])
    aux[2] = area / (dxc * dyc)
    x = xlo + (np.arange(1, mx + 1) - 0.5) * dxc
    y = ylo + (np.arange(1, my + 1) - 0.5) * dyc
    XC, YC = np.meshgrid(x, y, indexing="xy")
    xp, yp = mapc2p(XC, YC)
    A1, b1, x1, y1 = 1.0, 40.0, -0.5, 0.0
    A2, b2, x2, y2 = -1.0, 40.0, 0.5, 0.0
    q0 = np.zeros((1, my, mx))
    q0[0] = (A1 * np.exp(-b1 * ((xp - x1) ** 2 + (yp - y1) ** 2))
             + A2 * np.exp(-b2 * ((xp - x2) ** 2 + (yp - y2) ** 2)))
    return rd, "vc_advection_2d", {}, q0, aux


def random_acoustics_2d(mx, my, seed=0, bc=("extrap", "extrap", "extrap", "extrap"),
                        limiter="mc", order=2, trans=2, nout=1, tfinal=0.05):
    """Seeded random 2D acoustics state (smooth + noise) for parity tests on
    ragged sizes and every boundary-condition kind."""
    rng = np.random.default_rng(seed)
    rd, solver, params, _, _ = radial_acoustics_2d(n=8, nout=nout, tfinal=tfinal)
    cd = rd.clawdata
    cd.num_cells = [mx, my]
    cd.bc_lower = [bc[0], bc[2]]
    cd.bc_upper = [bc[1], bc[3]]
    cd.limiter = [limiter, limiter]
    cd.order = order
    cd.transverse_waves = trans
    x, _ = _centres(-1.0, 1.0, mx)
    y, _ = _centres(-1.0, 1.0, my)
    X, Y = np.meshgrid(x, y, indexing="xy")
    q0 = np.zeros((3, my, mx))
    q0[0] = 1.0 + np.exp(-20.0 * ((X - 0.2) ** 2 + (Y + 0.1) ** 2)) + 0.1 * rng.standard_normal((my, mx))
    q0[1] = 0.2 * rng.standard_normal((my, mx))
    q0[2] = 0.2 * rng.standard_normal((my, mx))
    return rd, solver, params, q0, None


# ------------------------------------------------------------------- 3D ---
def _two_layer_aux(mx, my, mz, zlower, dz, below, above):
    """aux[maux=2][mz+4][my+4][mx+4] = (Z, c) by the sign of the cell-centre z,
    ghost cells included (examples/acoustics_3d_heterogeneous/setaux.f)."""
    k = np.arange(-1, mz + 3, dtype=np.float64)
    zcell = zlower + (k - 0.5) * dz
    lower = zcell < 0.0
    aux = np.empty((2, mz + 4, my + 4, mx + 4))
    for m in range(2):
        aux[m] = np.where(lower, below[m], above[m])[:, None, None]
    return aux


def acoustics_3d_heterogeneous(n=20, nout=2, tfinal=1.0):
    """examples/acoustics_3d_heterogeneous (setrun.py, setprob.f, setaux.f,
    qinit.f, bc3.f) with the regression test's overrides
    (test_acoustics_3d_heterogeneous.py:17-19): (Z, c) = (2, 2) below z=0 and
    (1, 1) above, q0 = 0, van Leer, transverse_waves 22, and the piston wall
    ('user' BC) at z-upper driving the flow."""
    rd = ClawRunData("classic", 3)
    pd = rd.new_UserData("probdata", "setprob.data")
    for k, v in (("z1", 2.0), ("c1", 2.0), ("z2", 1.0), ("c2", 1.0)):
        pd.add_param(k, v)
    cd = rd.clawdata
    cd.lower, cd.upper, cd.num_cells = [-1.0] * 3, [1.0] * 3, [n, n, n]
    cd.num_eqn, cd.num_aux, cd.capa_index = 4, 2, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = True
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, 0.01, 1e9
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 50000
    cd.order, cd.transverse_waves, cd.dimensional_split = 2, 22, "unsplit"
    cd.num_waves, cd.limiter = 2, [3, 3]
    cd.bc_lower = ["extrap", "extrap", "extrap"]
    cd.bc_upper = ["extrap", "extrap", "user"]
    dz = 2.0 / float(np.float32(n))
    aux = _two_layer_aux(n, n, n, -1.0, dz, (2.0, 2.0), (1.0, 1.0))
    q0 = np.zeros((4, n, n, n))
    return rd, "vc_acoustics_3d", {}, q0, aux


def heterogeneous_acoustics_3d(n=256, nout=8, tfinal=0.8, limiter="mc", dt_initial=0.01,
                               shape=None):
    """3D heterogeneous acoustics workload: two layers split at z=0 (rho=1,
    K=1 below; rho=4, K=2 above; Z = sqrt(rho K), c = sqrt(K/rho) per cell),
    [-1,1]^3 with n^3 cells (or `shape` = (mx, my, mz)), Gaussian pulse
    p0 = exp(-80 |x - x0|^2) at x0 = (0, 0, -0.4), zero velocity; order 2,
    transverse_waves 22, MC, cfl 0.9, wall at z-lower, extrapolation
    elsewhere, t_final 0.8."""
    mx, my, mz = shape if shape is not None else (n, n, n)
    rd = ClawRunData("classic", 3)
    cd = rd.clawdata
    cd.lower, cd.upper, cd.num_cells = [-1.0] * 3, [1.0] * 3, [mx, my, mz]
    cd.num_eqn, cd.num_aux, cd.capa_index = 4, 2, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = True
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, dt_initial, 1e99
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 50000
    cd.order, cd.transverse_waves, cd.dimensional_split = 2, 22, "unsplit"
    cd.num_waves, cd.limiter = 2, [limiter, limiter]
    cd.bc_lower = ["extrap", "extrap", "wall"]
    cd.bc_upper = ["extrap", "extrap", "extrap"]
    x, _ = _centres(-1.0, 1.0, mx)
    y, _ = _centres(-1.0, 1.0, my)
    z, dz = _centres(-1.0, 1.0, mz)
    below = (np.sqrt(1.0 * 1.0), np.sqrt(1.0 / 1.0))
    above = (np.sqrt(4.0 * 2.0), np.sqrt(2.0 / 4.0))
    aux = _two_layer_aux(mx, my, mz, -1.0, dz, below, above)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    q0 = np.zeros((4, mz, my, mx))
    q0[0] = np.exp(-80.0 * (X * X + Y * Y + (Z + 0.4) ** 2))
    return rd, "vc_acoustics_3d", {}, q0, aux


def random_acoustics_3d(mx, my, mz, seed=0, bc=("extrap",) * 6, limiter="mc", trans=22,
                        order=2, nout=1, tfinal=0.02):
    """Seeded random 3D heterogeneous acoustics state (random per-cell (Z, c)
    and random q) for parity tests on ragged sizes and every BC kind."""
    rng = np.random.default_rng(seed)
    rd, solver, params, _, _ = heterogeneous_acoustics_3d(shape=(mx, my, mz), nout=nout,
                                                          tfinal=tfinal, limiter=limiter)
    cd = rd.clawdata
    cd.bc_lower = [bc[0], bc[2], bc[4]]
    cd.bc_upper = [bc[1], bc[3], bc[5]]
    cd.transverse_waves = trans
    cd.order = order
    aux = np.empty((2, mz + 4, my + 4, mx + 4))
    aux[0] = rng.uniform(0.5, 2.0, aux[0].shape)
    aux[1] = rng.uniform(0.5, 1.5, aux[1].shape)
    q0 = np.empty((4, mz, my, mx))
    q0[0] = 1.0 + 0.3 * rng.standard_normal((mz, my, mx))
    q0[1:] = 0.2 * rng.standard_normal((3, mz, my, mx))
    return rd, solver, params, q0, aux


# ------------------------------------------------------------- 2D Euler ---
def euler_quadrant_state(seed):
    """Seeded four-quadrant Riemann data: per quadrant rho ~ U[0.5, 2],
    p ~ U[0.1, 1.5], u, v ~ U[-0.75, 0.75]; split point ~ U[0.3, 0.7]^2.
    Returns (x_split, y_split, prim[4 quadrants][rho, u, v, p]) with the
    quadrants ordered (x < xs, y < ys), (x >= xs, y < ys), (x < xs, y >= ys),
    (x >= xs, y >= ys)."""
    rng = np.random.default_rng(seed)
    prim = np.empty((4, 4))
    for k in range(4):
        prim[k, 0] = rng.uniform(0.5, 2.0)
        prim[k, 3] = rng.uniform(0.1, 1.5)
        prim[k, 1] = rng.uniform(-0.75, 0.75)
        prim[k, 2] = rng.uniform(-0.75, 0.75)
    xs, ys = rng.uniform(0.3, 0.7, size=2)
    return float(xs), float(ys), prim


def euler_quadrants(n=256, seed=0, gamma=1.4, tfinal=0.25, nout=1, dt_initial=1e-3,
                    limiter="mc", order=2, trans=2, bc=("extrap",) * 4, shape=None):
    """One instance of the batched Euler workload: gamma = 1.4, Roe solver with
    the Harten-Hyman entropy fix, four-quadrant Riemann data on [0,1]^2 from
    `seed` (euler_quadrant_state), n^2 cells (or shape = (mx, my)); order 2,
    MC, transverse 2, extrapolation BCs, t_final 0.25."""
    mx, my = shape if shape is not None else (n, n)
    rd = ClawRunData("classic", 2)
    pd = rd.new_UserData("probdata", "setprob.data")
    pd.add_param("gamma", gamma)
    cd = rd.clawdata
    cd.lower, cd.upper, cd.num_cells = [0.0, 0.0], [1.0, 1.0], [mx, my]
    cd.num_eqn, cd.num_aux, cd.capa_index = 4, 0, 0
    cd.t0, cd.output_style, cd.num_output_times, cd.tfinal = 0.0, 1, nout, tfinal
    cd.output_t0 = True
    cd.dt_variable, cd.dt_initial, cd.dt_max = True, dt_initial, 1e99
    cd.cfl_desired, cd.cfl_max, cd.steps_max = 0.9, 1.0, 50000
    cd.order, cd.transverse_waves, cd.dimensional_split = order, trans, "unsplit"
    cd.num_waves, cd.limiter = 3, [limiter] * 3
    cd.bc_lower, cd.bc_upper = [bc[0], bc[2]], [bc[1], bc[3]]
    xs, ys, prim = euler_quadrant_state(seed)
    x, _ = _centres(0.0, 1.0, mx)
    y, _ = _centres(0.0, 1.0, my)
    X, Y = np.meshgrid(x, y, indexing="xy")
    quad = (X >= xs).astype(int) + 2 * (Y >= ys).astype(int)
    rho, u, v, p = (prim[quad, k] for k in range(4))
    q0 = np.empty((4, my, mx))
    q0[0] = rho
    q0[1] = rho * u
    q0[2] = rho * v
    q0[3] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return rd, "euler_roe_2d", {"gamma": gamma}, q0, None


def euler_ensemble_sizes(count=256, seed=0, nmin=128, nmax=1024):
    """Grid sides of the batched workload: N = round(exp(U[ln nmin, ln nmax]))
    per instance (log-uniform), from one seeded generator."""
    rng = np.random.default_rng(seed)
    return [int(round(float(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))) for _ in range(count)]
