"""ORACLE — test infrastructure only.

ctypes wrapper of the CPU restatement in claw_oracle.cpp, plus the
claw{1,2,3}ez frame loop (src/2d/claw2ez.f:265-324, src/1d/claw1ez.f,
src/3d/claw3ez.f) around it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs
use this module, always as the checker or the timed CPU reference.

Arrays cross in the product's SoA layout (q: [meqn]([mz])[my][mx] interior
cells; aux: [maux]([mz+4])[my+4][mx+4]) and are converted here to the
reference's Fortran layout q(meqn, 1-mbc:mx+mbc, 1-mbc:my+mbc(, 1-mbc:mz+mbc)).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "build")

SOLVER_IDS = {
    "acoustics_2d": 1,
    "vc_advection_2d": 2,
    "euler_roe_2d": 3,
    "acoustics_1d": 11,
    "vc_acoustics_1d": 12,
    "advection_1d": 13,
    "euler_roe_1d": 14,
    "vc_acoustics_3d": 21,
}
SOLVER_PARAMS = {
    "acoustics_2d": ("rho", "bulk"),
    "acoustics_1d": ("rho", "bulk"),
    "euler_roe_2d": ("gamma",),
    "advection_1d": ("u",),
    "euler_roe_1d": ("gamma",),
}

# bc code of the restated user BC (examples/acoustics_3d_heterogeneous/bc3.f:282-312)
PISTON_BC = 10
# restated source routines (examples/acoustics_2d_radial/1drad/src1.f:18-23)
SOURCE_IDS = {"radial": 1}
# restated before-step routines (edge velocities times cos(pi t / T))
B4STEP_IDS = {"reversing": 1}

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def build(quiet: bool = True):
    """Compile the oracle libraries with make (g++)."""
    subprocess.run(["make", "-C", HERE], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _load(variant: str):
    name = "liboracle.so" if variant == "parity" else "liboracle_fast.so"
    path = os.path.join(BUILD, name)
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    lib.orc_set_threads.argtypes = [ctypes.c_int]
    lib.orc_set_threads.restype = ctypes.c_int
    lib.orc_set_solver.argtypes = [ctypes.c_int, _D, ctypes.c_int]
    lib.orc_set_solver.restype = ctypes.c_int
    lib.orc_set_source.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
    lib.orc_set_source.restype = ctypes.c_int
    lib.orc_set_b4step.argtypes = [ctypes.c_int, ctypes.c_double]
    lib.orc_set_b4step.restype = ctypes.c_int
    lib.orc_b4step2.argtypes = [ctypes.c_int, ctypes.c_longlong, _D, _D, ctypes.c_double]
    lib.orc_b4step2.restype = ctypes.c_int
    lib.orc_claw2.argtypes = [ctypes.c_int] * 6 + [_D, _D, ctypes.c_double, ctypes.c_double,
                                                   ctypes.c_double, _D, _D, _D, _I, _I, _I, _I,
                                                   ctypes.c_int]
    lib.orc_claw2.restype = ctypes.c_int
    lib.orc_step2.argtypes = [ctypes.c_int] * 6 + [_D, _D, _D, ctypes.c_double, ctypes.c_double,
                                                   ctypes.c_double, _I, _I, ctypes.c_int, _D]
    lib.orc_step2.restype = ctypes.c_int
    lib.orc_bc2.argtypes = [ctypes.c_int] * 4 + [_D, _I]
    lib.orc_bc2.restype = ctypes.c_int
    lib.orc_claw1.argtypes = [ctypes.c_int] * 5 + [_D, _D, ctypes.c_double, ctypes.c_double, _D,
                                                   _D, _D, _I, _I, _I, _I, ctypes.c_int]
    lib.orc_claw1.restype = ctypes.c_int
    lib.orc_step1.argtypes = [ctypes.c_int] * 5 + [_D, _D, ctypes.c_double, ctypes.c_double, _I,
                                                   _I, ctypes.c_int, _D]
    lib.orc_step1.restype = ctypes.c_int
    lib.orc_bc1.argtypes = [ctypes.c_int] * 3 + [_D, _I]
    lib.orc_bc1.restype = ctypes.c_int
    lib.orc_claw3.argtypes = [ctypes.c_int] * 7 + [_D, _D] + [ctypes.c_double] * 6 + [
        _D, _D, _D, _I, _I, _I, _I, ctypes.c_int]
    lib.orc_claw3.restype = ctypes.c_int
    lib.orc_step3.argtypes = [ctypes.c_int] * 7 + [_D, _D, _D] + [ctypes.c_double] * 4 + [
        _I, _I, ctypes.c_int, _D]
    lib.orc_step3.restype = ctypes.c_int
    lib.orc_bc3.argtypes = [ctypes.c_int] * 5 + [_D, _I] + [ctypes.c_double] * 5
    lib.orc_bc3.restype = ctypes.c_int
    lib.orc_dimsp2.argtypes = [ctypes.c_int] * 6 + [_D, _D, _D, ctypes.c_double, ctypes.c_double,
                                                    ctypes.c_double, _I, _I, _D, ctypes.c_int, _D]
    lib.orc_dimsp2.restype = ctypes.c_int
    lib.orc_dimsp3.argtypes = [ctypes.c_int] * 7 + [_D, _D, _D] + [ctypes.c_double] * 4 + [
        _I, _I, _D, ctypes.c_int, _D]
    lib.orc_dimsp3.restype = ctypes.c_int
    return lib


def _p(a, t=_D):
    return a.ctypes.data_as(t)


def _codes(cd):
    """method(1:7), mthlim, mthbc from a ClawInputData."""
    nd = int(cd.num_dim)
    method = np.zeros(7, dtype=np.int32)
    method[0] = 1 if cd.dt_variable else 0
    method[1] = int(cd.order)
    method[2] = cd.transverse_code() if nd > 1 else 0
    split = cd.split_code() if nd > 1 else 0
    if split > 0:
        # src/2d/claw2ez.f:126 (-1 Godunov, -2 Strang); src/3d/claw3ez.f:136 (always -1)
        method[2] = -split if nd == 2 else -1
    method[3] = int(cd.verbosity)
    method[4] = cd.source_code()
    method[5] = int(cd.capa_index)
    method[6] = int(cd.num_aux)
    mthlim = np.array(cd.limiter_codes(), dtype=np.int32)
    lo, hi = cd.bc_codes()
    if nd == 1:
        mthbc = np.array([lo[0], hi[0]], dtype=np.int32)
    elif nd == 2:
        mthbc = np.array([lo[0], hi[0], lo[1], hi[1]], dtype=np.int32)
    else:
        mthbc = np.array([lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]], dtype=np.int32)
        if mthbc[5] == 0:
            # 'user' at z-upper: the piston wall of examples/acoustics_3d_heterogeneous
            mthbc[5] = PISTON_BC
    return method, mthlim, mthbc


class OracleGrid:
    """Reference-layout state of one grid driven by the CPU restatement."""

    def __init__(self, cd, solver: str, params: dict | None = None, variant: str = "parity",
                 user_source: str | None = None, user_b4step: str | None = None):
        self.lib = _load(variant)
        self.cd = cd
        self.nd = int(cd.num_dim)
        self.solver = solver
        self.meqn = int(cd.num_eqn)
        self.mwaves = int(cd.num_waves)
        self.maux = int(cd.num_aux)
        self.mbc = int(cd.num_ghost)
        self.cells = [int(n) for n in cd.num_cells][: self.nd]
        # dx = (upper - lower)/float(mx), float() being single precision
        self.dxs = [(float(cd.upper[d]) - float(cd.lower[d])) / float(np.float32(self.cells[d]))
                    for d in range(self.nd)]
        self.method, self.mthlim, self.mthbc = _codes(cd)
        self.use_fwaves = 1 if cd.use_fwaves else 0
        params = params or {}
        pv = np.array([float(params[k]) for k in SOLVER_PARAMS.get(solver, ())] or [0.0])
        self.pv = pv
        # the example's src routine (0 = the reference's default no-op)
        self.src = SOURCE_IDS[user_source] if user_source is not None else 0
        self.src_ndim = int(params.get("ndim", 2))
        self.b4 = B4STEP_IDS[user_b4step] if user_b4step is not None else 0
        self.b4_period = float(params.get("period", 1.0))
        g = tuple(n + 2 * self.mbc for n in reversed(self.cells))  # (my+4, mx+4) C order
        self.qf = np.zeros(g + (self.meqn,), dtype=np.float64)
        self.af = np.zeros(g + (max(self.maux, 1),), dtype=np.float64)
        self._set_solver()

    def _set_solver(self):
        self.lib.orc_set_solver(SOLVER_IDS[self.solver], _p(self.pv), len(self.pv))
        self.lib.orc_set_source(self.src, self.src_ndim, float(self.cd.lower[0]))
        self.lib.orc_set_b4step(self.b4, self.b4_period)

    def _interior(self):
        b = self.mbc
        return tuple(slice(b, -b) for _ in self.cells)

    def set_q(self, q):
        q = np.asarray(q, dtype=np.float64)
        self.qf[self._interior()] = np.moveaxis(q, 0, -1)

    def get_q(self):
        # a copy: with one field the moved view already counts as contiguous
        return np.array(np.moveaxis(self.qf[self._interior()], -1, 0), order="C", copy=True)

    def set_aux(self, aux):
        if self.maux:
            self.af[...] = np.moveaxis(np.asarray(aux, dtype=np.float64), 0, -1)

    def _cflv(self):
        return np.array([float(self.cd.cfl_max), float(self.cd.cfl_desired), 0.0, 0.0])

    def advance(self, tstart, tend, dt_initial):
        """claw{1,2}: returns (info, stats dict)."""
        self._set_solver()
        dtv = np.array([dt_initial, float(self.cd.dt_max), 0.0, 0.0, 0.0])
        cflv = np.array([float(self.cd.cfl_max), float(self.cd.cfl_desired), 0.0, 0.0])
        nv = np.array([int(self.cd.steps_max), 0], dtype=np.int32)
        te = ctypes.c_double(tend)
        if self.nd == 2:
            mx, my = self.cells
            info = self.lib.orc_claw2(self.meqn, self.mwaves, self.maux, self.mbc, mx, my,
                                      _p(self.qf), _p(self.af), self.dxs[0], self.dxs[1],
                                      float(tstart), ctypes.byref(te), _p(dtv), _p(cflv),
                                      _p(nv, _I), _p(self.method, _I), _p(self.mthlim, _I),
                                      _p(self.mthbc, _I), self.use_fwaves)
        elif self.nd == 1:
            (mx,) = self.cells
            info = self.lib.orc_claw1(self.meqn, self.mwaves, self.maux, self.mbc, mx,
                                      _p(self.qf), _p(self.af), self.dxs[0], float(tstart),
                                      ctypes.byref(te), _p(dtv), _p(cflv), _p(nv, _I),
                                      _p(self.method, _I), _p(self.mthlim, _I),
                                      _p(self.mthbc, _I), self.use_fwaves)
        else:
            mx, my, mz = self.cells
            info = self.lib.orc_claw3(self.meqn, self.mwaves, self.maux, self.mbc, mx, my, mz,
                                      _p(self.qf), _p(self.af), float(self.cd.lower[0]),
                                      float(self.cd.lower[1]), self.dxs[0], self.dxs[1],
                                      self.dxs[2], float(tstart), ctypes.byref(te), _p(dtv),
                                      _p(cflv), _p(nv, _I), _p(self.method, _I),
                                      _p(self.mthlim, _I), _p(self.mthbc, _I), self.use_fwaves)
        stats = dict(t_reached=te.value, dt_min=dtv[2], dt_max_taken=dtv[3], dt_next=dtv[4],
                     cfl_max_seen=cflv[2], cfl_last=cflv[3], steps_taken=int(nv[1]), info=info)
        return info, stats

    def step(self, dt, t=0.0):
        """bc + copy + one step1/2/3 of length dt (t: the bc time); returns cfl."""
        self._set_solver()
        cfl = ctypes.c_double(0.0)
        if self.nd == 2:
            mx, my = self.cells
            self.lib.orc_bc2(self.meqn, self.mbc, mx, my, _p(self.qf), _p(self.mthbc, _I))
            qold = self.qf.copy()
            af = self.af
            if self.b4:  # b4step2 at the step's start time, from the unscaled aux
                af = np.empty_like(self.af)
                self.lib.orc_b4step2(self.maux, self.af.size // max(self.maux, 1), _p(self.af),
                                     _p(af), float(t))
            if self.method[2] >= 0:
                rc = self.lib.orc_step2(self.meqn, self.mwaves, self.maux, self.mbc, mx, my,
                                        _p(qold), _p(self.qf), _p(af), self.dxs[0],
                                        self.dxs[1], float(dt), _p(self.method, _I),
                                        _p(self.mthlim, _I), self.use_fwaves, ctypes.byref(cfl))
            else:
                rc = self.lib.orc_dimsp2(self.meqn, self.mwaves, self.maux, self.mbc, mx, my,
                                         _p(qold), _p(self.qf), _p(af), self.dxs[0],
                                         self.dxs[1], float(dt), _p(self.method, _I),
                                         _p(self.mthlim, _I), _p(self._cflv()), self.use_fwaves,
                                         ctypes.byref(cfl))
        elif self.nd == 3:
            mx, my, mz = self.cells
            self.lib.orc_bc3(self.meqn, self.mbc, mx, my, mz, _p(self.qf), _p(self.mthbc, _I),
                             float(t), float(self.cd.lower[0]), float(self.cd.lower[1]),
                             self.dxs[0], self.dxs[1])
            qold = self.qf.copy()
            if self.method[2] >= 0:
                rc = self.lib.orc_step3(self.meqn, self.mwaves, self.maux, self.mbc, mx, my, mz,
                                        _p(qold), _p(self.qf), _p(self.af), self.dxs[0],
                                        self.dxs[1], self.dxs[2], float(dt), _p(self.method, _I),
                                        _p(self.mthlim, _I), self.use_fwaves, ctypes.byref(cfl))
            else:
                rc = self.lib.orc_dimsp3(self.meqn, self.mwaves, self.maux, self.mbc, mx, my, mz,
                                         _p(qold), _p(self.qf), _p(self.af), self.dxs[0],
                                         self.dxs[1], self.dxs[2], float(dt),
                                         _p(self.method, _I), _p(self.mthlim, _I),
                                         _p(self._cflv()), self.use_fwaves, ctypes.byref(cfl))
        else:
            (mx,) = self.cells
            self.lib.orc_bc1(self.meqn, self.mbc, mx, _p(self.qf), _p(self.mthbc, _I))
            rc = self.lib.orc_step1(self.meqn, self.mwaves, self.mbc, self.maux, mx, _p(self.qf),
                                    _p(self.af), self.dxs[0], float(dt), _p(self.method, _I),
                                    _p(self.mthlim, _I), self.use_fwaves, ctypes.byref(cfl))
        if rc != 0:
            raise RuntimeError(f"oracle step failed ({rc})")
        return cfl.value


def run_oracle(rundata, solver, params, q0, aux=None, variant="parity", flush_tiny=True,
               user_source=None, user_b4step=None):
    """claw{1,2}ez frame loop on the oracle; returns [(frame, t, q, stats)]."""
    cd = getattr(rundata, "clawdata", rundata)
    g = OracleGrid(cd, solver, params, variant, user_source, user_b4step)
    q = np.array(q0, dtype=np.float64, copy=True)
    if flush_tiny:
        q[np.abs(q) < 1e-99] = 0.0
    g.set_q(q)
    if aux is not None:
        g.set_aux(aux)
    frames = []
    t0 = float(cd.t0)
    if cd.output_t0:
        frames.append((0, t0, q.copy(), {}))
    style = int(cd.output_style)
    if style == 1:
        nout, nstepout = int(cd.num_output_times), 1
        dtout = (float(cd.tfinal) - t0) / float(np.float32(nout))
    elif style == 2:
        nout, nstepout = len(cd.output_times), 1
    else:
        nout, nstepout = int(cd.total_steps), int(cd.output_step_interval)
    tend = t0
    dt = float(cd.dt_initial)
    for n in range(1, nout + 1):
        tstart = tend
        if style == 1:
            tend = tstart + dtout
        elif style == 2:
            tend = float(cd.output_times[n - 1])
        else:
            tend = tstart - 1.0
        info, st = g.advance(tstart, tend, dt)
        if info != 0:
            raise RuntimeError(f"oracle claw returned info={info}")
        dt = st["dt_next"]
        tend = st["t_reached"]
        if (n // nstepout) * nstepout == n:
            qn = g.get_q()
            if flush_tiny:
                tiny = np.abs(qn) < 1e-99
                if tiny.any():
                    qn[tiny] = 0.0
                    g.set_q(qn)
            frames.append((n // nstepout, tend, qn, st))
    return frames
