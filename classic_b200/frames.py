"""fort.qNNNN / fort.tNNNN frame files in the reference's ASCII format.

Writer: src/2d/out2.f:20-111 (1D: src/1d/out1.f; 3D: src/3d/out3.f).  Values are written with
Fortran ``e26.16`` (16 significant digits in 0.d...dE+ee form) after the
in-place flush of |q| < 1e-99 (src/2d/out2.f:70); the header carries grid
number, AMR level, mx, my, xlow, ylow, dx, dy, and fort.t carries time, meqn,
ngrids, maux, ndim, nghost and the format name.  ``read_frame`` parses a
frame back (the restart path of src/2d/restart2.f reads the same layout).
fort.info gets one record per output frame with the claw call's dt / CFL /
step returns (``start_info``, ``append_info``).
"""
from __future__ import annotations

import os

import numpy as np


def fortran_e(v: float, w: int = 26, d: int = 16) -> str:
    """Fortran Ew.d edit descriptor (gfortran form, leading '0.')."""
    v = float(v)
    if v == 0.0 or not np.isfinite(v):
        if v == 0.0:
            s = "0." + "0" * d + "E+00"
            if np.signbit(v):
                s = "-" + s
            return s.rjust(w)
        return ("NaN" if np.isnan(v) else ("-Infinity" if v < 0 else "Infinity")).rjust(w)
    mant, exp = f"{abs(v):.{d - 1}e}".split("e")
    digits = mant.replace(".", "")
    e10 = int(exp) + 1
    es = f"{'+' if e10 >= 0 else '-'}{abs(e10):02d}"
    if abs(e10) > 99:
        s = f"0.{digits}{'+' if e10 >= 0 else '-'}{abs(e10):03d}"
    else:
        s = f"0.{digits}E{es}"
    if v < 0:
        s = "-" + s
    return s.rjust(w)


def _i5(n: int) -> str:
    return f"{n:5d}"


def fortran_d(v: float, w: int = 15, d: int = 4) -> str:
    """Fortran Dw.d edit descriptor (gfortran form: 0.dddD+ee)."""
    return fortran_e(v, w, d).replace("E", "D")


def fortran_i(n: int, w: int) -> str:
    """Fortran Iw: right-justified, or w asterisks when the value does not fit."""
    s = str(int(n))
    return s.rjust(w) if len(s) <= w else "*" * w


def start_info(outdir: str) -> str:
    """Create (truncate) fort.info, as claw2ez opens it with status='unknown'
    at the start of a run (src/2d/claw2ez.f:34; claw1ez.f:28, claw3ez.f:46)."""
    path = os.path.join(outdir, "fort.info")
    open(path, "w").close()
    return path


def append_info(outdir: str, tend: float, info: int, stats: dict) -> None:
    """Append one output frame's record to fort.info: claw2ez's format 1010
    (src/2d/claw2ez.f:308-309, 319-322) with dtv(3:5), cflv(3:4) and nv(2)
    of the claw call that reached the frame."""
    rec = ("tend =" + fortran_d(tend) + "\n"
           "info =" + fortran_i(info, 5) + "\n"
           "smallest dt =" + fortran_d(stats["dt_min"]) + "\n"
           "largest dt =" + fortran_d(stats["dt_max_taken"]) + "\n"
           "last dt =" + fortran_d(stats["dt_next"]) + "\n"
           "largest cfl =" + fortran_d(stats["cfl_max_seen"]) + "\n"
           "last cfl =" + fortran_d(stats["cfl_last"]) + "\n"
           "steps taken =" + fortran_i(stats["steps_taken"], 4) + "\n\n")
    with open(os.path.join(outdir, "fort.info"), "a") as f:
        f.write(rec)


def flush_tiny(q: np.ndarray) -> np.ndarray:
    q = np.array(q, dtype=np.float64, copy=True)
    q[np.abs(q) < 1e-99] = 0.0
    return q


def write_frame(outdir: str, frame: int, t: float, q: np.ndarray, lower, dxs,
                maux: int = 0, nghost: int = 2) -> tuple[str, str]:
    """Write fort.qNNNN and fort.tNNNN for a 1D, 2D or 3D grid (q: [meqn]([mz])([my])[mx])."""
    q = flush_tiny(q)
    meqn = q.shape[0]
    ndim = q.ndim - 1
    fq = os.path.join(outdir, f"fort.q{frame:04d}")
    ft = os.path.join(outdir, f"fort.t{frame:04d}")
    lines = [_i5(1) + "                 grid_number", _i5(1) + "                 AMR_level"]
    if ndim == 1:
        mx = q.shape[1]
        lines.append(_i5(mx) + "                 mx")
        lines.append(f"{float(lower[0]):18.8E}    xlow")
        lines.append(f"{float(dxs[0]):18.8E}    dx")
        lines.append("")
        for i in range(mx):
            lines.append("".join(fortran_e(q[m, i]) for m in range(meqn)))
        lines.append(" ")
        lines.append(" ")
    elif ndim == 3:
        mz, my, mx = q.shape[1], q.shape[2], q.shape[3]
        lines.append(_i5(mx) + "                 mx")
        lines.append(_i5(my) + "                 my")
        lines.append(_i5(mz) + "                 mz")
        for d, nm in enumerate(("xlow", "ylow", "zlow")):
            lines.append(fortran_e(lower[d]) + "    " + nm)
        for d, nm in enumerate(("dx", "dy", "dz")):
            lines.append(fortran_e(dxs[d]) + "    " + nm)
        lines.append("")
        for k in range(mz):
            for j in range(my):
                for i in range(mx):
                    lines.append("".join(fortran_e(q[m, k, j, i]) for m in range(meqn)))
                lines.append(" ")
            lines.append(" ")
        lines.append(" ")
    else:
        my, mx = q.shape[1], q.shape[2]
        lines.append(_i5(mx) + "                 mx")
        lines.append(_i5(my) + "                 my")
        lines.append(fortran_e(lower[0]) + "    xlow")
        lines.append(fortran_e(lower[1]) + "    ylow")
        lines.append(fortran_e(dxs[0]) + "    dx")
        lines.append(fortran_e(dxs[1]) + "    dy")
        lines.append("")
        for j in range(my):
            for i in range(mx):
                lines.append("".join(fortran_e(q[m, j, i]) for m in range(meqn)))
            lines.append(" ")
        lines.append(" ")
    with open(fq, "w") as f:
        f.write("\n".join(lines) + "\n")
    tl = [fortran_e(t) + "    time", _i5(meqn) + "                 meqn",
          _i5(1) + "                 ngrids", _i5(maux) + "                 maux",
          _i5(ndim) + "                 ndim", _i5(nghost) + "                 nghost",
          f"{'ascii':>10}                 format", "", ""]
    with open(ft, "w") as f:
        f.write("\n".join(tl) + "\n")
    return fq, ft


def read_frame(outdir: str, frame: int):
    """Read fort.qNNNN/fort.tNNNN back: returns (t, q[meqn]([mz])([my])[mx])."""
    with open(os.path.join(outdir, f"fort.t{frame:04d}")) as f:
        tl = f.read().split("\n")
    t = float(tl[0].split()[0].replace("D", "E"))
    meqn = int(tl[1].split()[0])
    ndim = int(tl[4].split()[0])
    with open(os.path.join(outdir, f"fort.q{frame:04d}")) as f:
        ql = f.read().split("\n")
    mx = int(ql[2].split()[0])
    mz = 1
    if ndim == 1:
        start, my = 6, 1
    elif ndim == 2:
        my = int(ql[3].split()[0])
        start = 9
    else:
        my = int(ql[3].split()[0])
        mz = int(ql[4].split()[0])
        start = 12
    vals = []
    for ln in ql[start:]:
        toks = ln.split()
        if toks:
            vals.extend(float(x.replace("D", "E")) for x in toks)
    a = np.array(vals, dtype=np.float64).reshape(mz * my * mx, meqn)
    if ndim == 1:
        return t, a.T.reshape(meqn, mx).copy()
    if ndim == 2:
        return t, a.T.reshape(meqn, my, mx).copy()
    return t, a.T.reshape(meqn, mz, my, mx).copy()
