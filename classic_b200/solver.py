"""Host-side mirror of the reference's driver layer.

``Solver`` wraps one handle of the C ABI (include/claw_b200.h): the device
state of one grid plus the claw2 analogue ``advance``.  ``run`` is the
claw{1,2}ez frame loop (src/2d/claw2ez.f:265-324): tend accumulates
``dtout`` per frame, the last dt of a frame seeds the next (dtv(1)=dtv(5),
src/2d/claw2ez.f:290), and each output frame applies out2's in-place flush
of |q| < 1e-99 (src/2d/out2.f:70) before the run continues.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np

from . import _lib
from ._lib import ClawConfig, ClawStats, SOLVER_IDS, PRECISIONS, check
from .data import ClawInputData, ClawRunData

# Problem parameters each solver reads (the setprob values), in C order.
SOLVER_PARAMS = {
    "acoustics_2d": ("rho", "bulk"),
    "acoustics_1d": ("rho", "bulk"),
    "euler_roe_2d": ("gamma",),
    "vc_advection_2d": (),
    "vc_acoustics_1d": (),
    "advection_1d": ("u",),
    "euler_roe_1d": ("gamma",),
    "vc_acoustics_3d": (),
}


# Built-in user boundary conditions ('user' in bc_lower / bc_upper), by name.
USER_BCS = {"piston": 10}  # examples/acoustics_3d_heterogeneous/bc3.f:282-312, z-upper
# Built-in source terms (the example's src1 / src2), by name; their parameters
# come from the problem parameters ("ndim").
USER_SOURCES = {"radial": 1}  # examples/acoustics_2d_radial/1drad/src1.f:18-23
# Built-in before-step routines (the example's b4step2), by name; parameter
# "period" of the problem parameters.
USER_B4STEPS = {"reversing": 1}  # edge velocities of vc_advection_2d times cos(pi t / T)


def make_config(cd: ClawInputData, solver: str, params: dict | None = None,
                precision: str = "fp64", user_bc: str | None = None,
                user_source: str | None = None, user_b4step: str | None = None) -> ClawConfig:
    """Map clawdata + solver choice onto the C ``claw_config``.  ``user_bc``
    names the built-in routine that stands for the example's own bc code
    wherever clawdata says 'user'; ``user_source`` the built-in routine that
    stands for the example's src1 / src2 (applied as clawdata.source_split
    says; without one the source step is the reference's default no-op);
    ``user_b4step`` the one that stands for its b4step2 (default: nothing)."""
    if solver not in SOLVER_IDS:
        raise ValueError(f"unknown solver {solver!r}; built: {sorted(SOLVER_IDS)}")
    params = params or {}
    c = ClawConfig()
    nd = int(cd.num_dim)
    c.num_dim = nd
    for d in range(3):
        c.num_cells[d] = int(cd.num_cells[d]) if d < nd else 1
        c.lower[d] = float(cd.lower[d]) if d < nd else 0.0
        c.upper[d] = float(cd.upper[d]) if d < nd else 1.0
    c.num_eqn = int(cd.num_eqn)
    c.num_waves = int(cd.num_waves)
    c.num_aux = int(cd.num_aux)
    c.capa_index = int(cd.capa_index)
    c.dt_variable = 1 if cd.dt_variable else 0
    c.order = int(cd.order)
    c.transverse_waves = cd.transverse_code() if nd > 1 else 0
    c.dimensional_split = cd.split_code() if nd > 1 else 0
    c.verbosity = int(cd.verbosity)
    c.source_split = cd.source_code()
    if user_source is not None:
        if user_source not in USER_SOURCES:
            raise ValueError(f"unknown user_source {user_source!r}; built: {sorted(USER_SOURCES)}")
        c.source_id = USER_SOURCES[user_source]
        c.source_ndim = int(params.get("ndim", 2))
    if user_b4step is not None:
        if user_b4step not in USER_B4STEPS:
            raise ValueError(f"unknown user_b4step {user_b4step!r}; built: {sorted(USER_B4STEPS)}")
        c.b4step_id = USER_B4STEPS[user_b4step]
        c.b4step_param = float(params.get("period", 1.0))
    c.use_fwaves = 1 if cd.use_fwaves else 0
    lim = cd.limiter_codes()
    if len(lim) != c.num_waves:
        raise ValueError(f"{len(lim)} limiters for {c.num_waves} waves")
    for k, v in enumerate(lim):
        c.limiter[k] = v
    c.num_ghost = int(cd.num_ghost)
    lo, hi = cd.bc_codes()
    if user_bc is not None:
        if user_bc not in USER_BCS:
            raise ValueError(f"unknown user_bc {user_bc!r}; built: {sorted(USER_BCS)}")
        lo = [USER_BCS[user_bc] if v == 0 else v for v in lo]
        hi = [USER_BCS[user_bc] if v == 0 else v for v in hi]
    for d in range(3):
        c.bc_lower[d] = lo[d] if d < nd else 1
        c.bc_upper[d] = hi[d] if d < nd else 1
    c.dt_initial = float(cd.dt_initial)
    c.dt_max = float(cd.dt_max)
    c.cfl_max = float(cd.cfl_max)
    c.cfl_desired = float(cd.cfl_desired)
    c.steps_max = int(cd.steps_max)
    c.solver_id = SOLVER_IDS[solver]
    for k, name in enumerate(SOLVER_PARAMS.get(solver, ())):
        if name not in params:
            raise ValueError(f"solver {solver} needs parameter {name!r}")
        c.solver_params[k] = float(params[name])
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    c.precision = PRECISIONS[precision]
    return c


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Solver:
    """Device state of one grid and the step / advance entry points."""

    def __init__(self, clawdata, solver: str, params: dict | None = None,
                 precision: str = "fp64", user_bc: str | None = None,
                 user_source: str | None = None, user_b4step: str | None = None):
        if isinstance(clawdata, ClawRunData):
            clawdata = clawdata.clawdata
        self.lib = _lib.load()
        self.clawdata = clawdata
        self.solver = solver
        self.precision = precision
        self.cfg = make_config(clawdata, solver, params, precision, user_bc, user_source,
                               user_b4step)
        self.ndim = self.cfg.num_dim
        self.meqn = self.cfg.num_eqn
        self.maux = self.cfg.num_aux
        cells = [self.cfg.num_cells[d] for d in range(self.ndim)]
        self.q_shape = (self.meqn,) + tuple(reversed(cells))
        self.aux_shape = (self.maux,) + tuple(n + 4 for n in reversed(cells))
        h = ctypes.c_void_p()
        check(self.lib.claw_create(ctypes.byref(self.cfg), ctypes.byref(h)), "claw_create")
        self._h = h

    # -- state --------------------------------------------------------------
    def set_q(self, q: np.ndarray):
        q = np.ascontiguousarray(q, dtype=np.float64)
        if q.shape != self.q_shape:
            raise ValueError(f"q shape {q.shape} != {self.q_shape}")
        check(self.lib.claw_set_q(self._h, _dptr(q)), "claw_set_q")

    def get_q(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.q_shape, dtype=np.float64)
        check(self.lib.claw_get_q(self._h, _dptr(out)), "claw_get_q")
        return out

    def set_aux(self, aux: np.ndarray):
        aux = np.ascontiguousarray(aux, dtype=np.float64)
        if aux.shape != self.aux_shape:
            raise ValueError(f"aux shape {aux.shape} != {self.aux_shape}")
        check(self.lib.claw_set_aux(self._h, _dptr(aux)), "claw_set_aux")

    # -- stepping -----------------------------------------------------------
    def step(self, dt: float) -> float:
        """One step of length dt (bc + step2/step3); returns the Courant number."""
        cfl = ctypes.c_double(0.0)
        check(self.lib.claw_step(self._h, float(dt), ctypes.byref(cfl)), "claw_step")
        return cfl.value

    def advance(self, tstart: float, tend: float, dt_initial: float):
        """claw2: advance with dt control; returns (info, stats dict)."""
        st = ClawStats()
        info = check(self.lib.claw_advance(self._h, float(tstart), float(tend),
                                           float(dt_initial), ctypes.byref(st)), "claw_advance")
        return info, st.as_dict()

    def advance_host(self, q: np.ndarray, tstart: float, tend: float, dt_initial: float):
        """The whole claw2 call on a host array (q in, q out, in place)."""
        if q.dtype != np.float64 or not q.flags.c_contiguous or q.shape != self.q_shape:
            raise ValueError("q must be a C-contiguous float64 array of the grid's shape")
        st = ClawStats()
        info = check(self.lib.claw_advance_host(self._h, _dptr(q), float(tstart), float(tend),
                                                float(dt_initial), ctypes.byref(st)),
                     "claw_advance_host")
        return info, st.as_dict()

    def set_steps_max(self, n: int):
        """nv(1) of the following advance calls: return (info 11) after n steps."""
        check(self.lib.claw_set_steps_max(self._h, int(n)), "claw_set_steps_max")

    def launch_count(self) -> int:
        return int(self.lib.claw_launch_count(self._h))

    def totals(self) -> np.ndarray:
        """Conserved totals sum(capa * q_m) per field, FP64 compensated sums."""
        out = np.zeros(self.meqn)
        check(self.lib.claw_totals(self._h, _dptr(out)), "claw_totals")
        return out

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.claw_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclass
class Frame:
    frame: int
    t: float
    q: np.ndarray
    stats: dict = field(default_factory=dict)


def frame_times(cd: ClawInputData):
    """(nout, nstepout, tend generator) of claw2ez's output loop."""
    style = int(cd.output_style)
    if style == 1:
        return int(cd.num_output_times), 1
    if style == 2:
        return len(cd.output_times), 1
    if style == 3:
        return int(cd.total_steps), int(cd.output_step_interval)
    raise ValueError(f"bad output_style {style}")


def run(rundata, solver: str, params: dict | None, q0: np.ndarray | None,
        aux: np.ndarray | None = None, precision: str = "fp64",
        on_frame: Callable[[Frame], None] | None = None, keep_frames: bool = True,
        flush_tiny: bool = True, solver_obj: Solver | None = None, user_bc: str | None = None,
        outdir: str | None = None, user_source: str | None = None,
        user_b4step: str | None = None):
    """claw{1,2,3}ez's frame loop on the GPU.  Returns the list of frames
    (frame 0 included when output_t0); raises on a nonzero info.

    With ``outdir`` every output frame is also written as fort.qNNNN /
    fort.tNNNN (out2.f's format) and gets a fort.info record (the dt / CFL /
    step returns of the claw call that reached it), and a restart run (clawdata.restart)
    reads its q and start time from the frame clawdata.restart_file names in
    that directory and continues the frame numbering from it, as claw2ez does
    (src/2d/claw2ez.f:236-271; dtout keeps the data's t0)."""
    from . import frames as _frames
    cd = rundata.clawdata if isinstance(rundata, ClawRunData) else rundata
    s = solver_obj or Solver(cd, solver, params, precision, user_bc, user_source, user_b4step)
    nd = int(cd.num_dim)
    lower = [float(cd.lower[d]) for d in range(nd)]
    dxs = [(float(cd.upper[d]) - float(cd.lower[d])) / float(np.float32(int(cd.num_cells[d])))
           for d in range(nd)]
    rest = bool(getattr(cd, "restart", False))
    iframe0 = 0
    t0 = float(cd.t0)
    dtout0 = t0  # claw2ez computes dtout from the data's t0
    if rest:
        if outdir is None:
            raise ValueError("a restart run needs outdir holding the restart frame")
        iframe0 = int("".join(ch for ch in str(cd.restart_file) if ch.isdigit()) or 0)
        t0, q = _frames.read_frame(outdir, iframe0)
    else:
        q = np.array(q0, dtype=np.float64, copy=True)
    if flush_tiny:
        q[np.abs(q) < 1e-99] = 0.0
    s.set_q(q)
    if aux is not None:
        s.set_aux(aux)
    frames = []
    if outdir is not None:
        _frames.start_info(outdir)
    if not rest and (cd.output_t0 or int(cd.output_style) == 2):
        f0 = Frame(0, t0, q.copy())
        if outdir is not None:
            _frames.write_frame(outdir, 0, t0, q, lower, dxs, maux=int(cd.num_aux),
                                nghost=int(cd.num_ghost))
        if on_frame:
            on_frame(f0)
        if keep_frames:
            frames.append(f0)
    nout, nstepout = frame_times(cd)
    # dtout = (tfinal - t0)/float(nout), src/2d/claw2ez.f:197-199
    dtout = (float(cd.tfinal) - dtout0) / float(np.float32(nout)) if int(cd.output_style) == 1 else None
    tend = t0
    dt = float(cd.dt_initial)
    for n in range(iframe0 * nstepout + 1, nout + 1):
        tstart = tend
        style = int(cd.output_style)
        if style == 1:
            tend = tstart + dtout
        elif style == 2:
            tend = float(cd.output_times[n - 1])
        else:
            tend = tstart - 1.0
        info, st = s.advance(tstart, tend, dt)
        if info != 0:
            raise RuntimeError(f"claw advance returned info={info} (stats {st})")
        dt = st["dt_next"]
        tend = st["t_reached"]
        iframe = n // nstepout
        if iframe * nstepout == n:
            q = s.get_q()
            if flush_tiny:
                tiny = np.abs(q) < 1e-99
                if tiny.any():
                    q[tiny] = 0.0
                    s.set_q(q)
            fr = Frame(iframe, tend, q, st)
            if outdir is not None:
                _frames.write_frame(outdir, iframe, tend, q, lower, dxs, maux=int(cd.num_aux),
                                    nghost=int(cd.num_ghost))
                _frames.append_info(outdir, tend, info, st)
            if on_frame:
                on_frame(fr)
            if keep_frames:
                frames.append(fr)
    if solver_obj is None:
        s.close()
    return frames


class BatchSolver:
    """Many independent 2D grids of one solver and method (uneven sizes), each
    with its own claw2 dt control, advanced together (claw_batch_* of the C
    ABI): one persistent launch per step over the rows of every instance
    still running."""

    def __init__(self, clawdatas, solver: str, params: dict | None = None,
                 precision: str = "fp64"):
        """precision "fp64" (reference order) or "fp64_fma" (the contracted
        build: fused multiply-adds, Newton reciprocals and roots)."""
        self.lib = _lib.load()
        cds = [c.clawdata if isinstance(c, ClawRunData) else c for c in clawdatas]
        self.count = len(cds)
        arr = (ClawConfig * self.count)()
        self.q_shapes = []
        for k, cd in enumerate(cds):
            arr[k] = make_config(cd, solver, params, precision)
            cells = [arr[k].num_cells[d] for d in range(2)]
            self.q_shapes.append((arr[k].num_eqn, cells[1], cells[0]))
        self._cfgs = arr
        h = ctypes.c_void_p()
        check(self.lib.claw_batch_create(arr, self.count, ctypes.byref(h)), "claw_batch_create")
        self._h = h

    def set_q(self, k: int, q: np.ndarray):
        q = np.ascontiguousarray(q, dtype=np.float64)
        if q.shape != self.q_shapes[k]:
            raise ValueError(f"q shape {q.shape} != {self.q_shapes[k]}")
        check(self.lib.claw_batch_set_q(self._h, k, _dptr(q)), "claw_batch_set_q")

    def get_q(self, k: int) -> np.ndarray:
        out = np.empty(self.q_shapes[k], dtype=np.float64)
        check(self.lib.claw_batch_get_q(self._h, k, _dptr(out)), "claw_batch_get_q")
        return out

    def autotune(self, dt_trial=None, repeats: int = 3) -> dict:
        """Choose the batch launch shape (tile height in rows, CTAs per SM) by
        timing one step of every instance per candidate; the state is left as
        it was.  Returns the chosen shape and its time per step."""
        dts = None
        if dt_trial is not None:
            dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt_trial, dtype=np.float64),
                                                       (self.count,)))
        rows, ctas, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(self.lib.claw_batch_autotune(self._h, _dptr(dts) if dts is not None else None,
                                           int(repeats), ctypes.byref(rows), ctypes.byref(ctas),
                                           ctypes.byref(ms)), "claw_batch_autotune")
        return {"min_rows": rows.value, "ctas_per_sm": ctas.value, "ms_per_step": ms.value}

    def set_shape(self, min_rows: int, ctas_per_sm: int):
        check(self.lib.claw_batch_set_shape(self._h, int(min_rows), int(ctas_per_sm)),
              "claw_batch_set_shape")

    def advance(self, tstart: float, tend: float, dt_initial=None):
        """Advance every instance; returns (first nonzero info or 0, [stats])."""
        st = (ClawStats * self.count)()
        dts = None
        if dt_initial is not None:
            dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt_initial, dtype=np.float64),
                                                       (self.count,)))
        info = check(self.lib.claw_batch_advance(self._h, float(tstart), float(tend),
                                                 _dptr(dts) if dts is not None else None, st),
                     "claw_batch_advance")
        return info, [st[k].as_dict() for k in range(self.count)]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.claw_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
