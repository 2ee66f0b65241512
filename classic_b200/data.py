"""Drop-in for the parts of ``clawpack.clawutil.data`` that a Clawpack Classic
``setrun.py`` uses, so an existing ``setrun.py`` runs unchanged after
``from clawpack.clawutil import data`` is pointed here (see
``install_clawutil_alias``).

``ClawRunData(pkg, num_dim)`` carries ``.clawdata`` (a ``ClawInputData``)
and user data created by ``new_UserData(name, fname)`` / ``add_param``.
``write()`` produces ``claw.data`` in the order ``claw2ez`` reads it
(src/2d/claw2ez.f:39-156; claw1ez/claw3ez are the same with other
dimensions) and one file per user data block; ``read_claw_data`` parses it
back.  ``to_config`` maps the clawdata fields onto the C struct of
include/claw_b200.h, with the string-to-integer codes the reference's
setrun comments document (e.g. examples/acoustics_2d_radial/setrun.py:182-225).
"""
from __future__ import annotations

import os
import sys
import types
from collections import OrderedDict

LIMITERS = {"none": 0, "minmod": 1, "superbee": 2, "vanleer": 3, "van leer": 3, "mc": 4,
            "beam-warming": 5, "beamwarming": 5}
BCS = {"user": 0, "extrap": 1, "periodic": 2, "wall": 3}
TRANSVERSE = {"none": 0, "increment": 1, "all": 2}
SPLIT = {"unsplit": 0, "godunov": 1, "strang": 2, "none": 0}
SOURCE = {"none": 0, "godunov": 1, "strang": 2}


def _code(value, table, what):
    if isinstance(value, bool):
        return int(value)
    if isinstance(value, (int,)):
        return int(value)
    if isinstance(value, float) and value.is_integer():
        return int(value)
    key = str(value).strip().lower()
    if key not in table:
        raise ValueError(f"unknown {what} {value!r}; expected one of {sorted(table)}")
    return table[key]


class UserData:
    """Named problem parameters (``rundata.new_UserData``), written one per
    line as ``value  =: name  # description``."""

    def __init__(self, fname="setprob.data"):
        self._fname = fname
        self._params = OrderedDict()
        self._descr = {}

    def add_param(self, name, value, descr=""):
        self._params[name] = value
        self._descr[name] = descr
        setattr(self, name, value)

    def __getitem__(self, name):
        return getattr(self, name)

    @property
    def params(self):
        return OrderedDict((k, getattr(self, k)) for k in self._params)

    def write(self, path="."):
        with open(os.path.join(path, self._fname), "w") as f:
            for k in self._params:
                v = getattr(self, k)
                f.write(f"{_fmt(v):<30} =: {k}  # {self._descr.get(k, '')}\n")


class ClawInputData:
    """The ``clawdata`` object of ClawRunData with the reference's defaults."""

    def __init__(self, num_dim):
        self.num_dim = num_dim
        self.lower = [0.0] * num_dim
        self.upper = [1.0] * num_dim
        self.num_cells = [100] * num_dim
        self.num_eqn = 1
        self.num_aux = 0
        self.capa_index = 0
        self.t0 = 0.0
        self.restart = False
        self.restart_file = "fort.q0000"
        self.output_style = 1
        self.num_output_times = 10
        self.tfinal = 1.0
        self.output_t0 = True
        self.output_times = []
        self.output_step_interval = 1
        self.total_steps = 1
        self.output_format = "ascii"
        self.output_q_components = "all"
        self.output_aux_components = "none"
        self.output_aux_onlyonce = True
        self.verbosity = 0
        self.dt_variable = True
        self.dt_initial = 1e-5
        self.dt_max = 1e99
        self.cfl_desired = 0.9
        self.cfl_max = 1.0
        self.steps_max = 50000
        self.order = 2
        self.transverse_waves = 2 if num_dim == 2 else (22 if num_dim == 3 else 0)
        self.dimensional_split = "unsplit"
        self.num_waves = 1
        self.limiter = ["minmod"]
        self.use_fwaves = False
        self.source_split = 0
        self.num_ghost = 2
        self.bc_lower = ["extrap"] * num_dim
        self.bc_upper = ["extrap"] * num_dim

    # integer views -----------------------------------------------------
    def limiter_codes(self):
        return [_code(v, LIMITERS, "limiter") for v in self.limiter]

    def bc_codes(self):
        lo = [_code(v, BCS, "bc") for v in self.bc_lower]
        hi = [_code(v, BCS, "bc") for v in self.bc_upper]
        return lo, hi

    def transverse_code(self):
        return _code(self.transverse_waves, TRANSVERSE, "transverse_waves")

    def split_code(self):
        return _code(self.dimensional_split, SPLIT, "dimensional_split")

    def source_code(self):
        return _code(self.source_split, SOURCE, "source_split")


class ClawRunData:
    """``ClawRunData('classic', num_dim)``."""

    def __init__(self, pkg="classic", num_dim=2):
        if str(pkg).lower() != "classic":
            raise ValueError("only the 'classic' package is provided")
        self.pkg = "classic"
        self.num_dim = num_dim
        self.clawdata = ClawInputData(num_dim)
        self.data_list = [self.clawdata]
        self._user = OrderedDict()

    def new_UserData(self, name, fname):
        u = UserData(fname)
        self._user[name] = u
        setattr(self, name, u)
        self.data_list.append(u)
        return u

    @property
    def user_data(self):
        return self._user

    def write(self, path="."):
        write_claw_data(self.clawdata, os.path.join(path, "claw.data"))
        for u in self._user.values():
            u.write(path)


# ---------------------------------------------------------------- claw.data ---
def _fmt(v):
    if isinstance(v, bool):
        return "T" if v else "F"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        return repr(float(v))
    if isinstance(v, (list, tuple)):
        return " ".join(_fmt(x) for x in v)
    return str(v)


def write_claw_data(cd: ClawInputData, fname="claw.data"):
    """Write claw.data in claw2ez's read order (src/2d/claw2ez.f:39-156)."""
    lines = []

    def add(value, name):
        lines.append(f"{_fmt(value):<40} =: {name}")

    add(cd.num_dim, "num_dim")
    add([float(x) for x in cd.lower], "lower")
    add([float(x) for x in cd.upper], "upper")
    add([int(x) for x in cd.num_cells], "num_cells")
    add(int(cd.num_eqn), "num_eqn")
    add(int(cd.num_waves), "num_waves")
    add(int(cd.num_aux), "num_aux")
    add(float(cd.t0), "t0")
    add(int(cd.output_style), "output_style")
    if cd.output_style == 1:
        add(int(cd.num_output_times), "num_output_times")
        add(float(cd.tfinal), "tfinal")
        add(bool(cd.output_t0), "output_t0")
    elif cd.output_style == 2:
        add(len(cd.output_times), "num_output_times")
        add([float(t) for t in cd.output_times], "output_times")
    elif cd.output_style == 3:
        add(int(cd.output_step_interval), "output_step_interval")
        add(int(cd.total_steps), "total_steps")
        add(bool(cd.output_t0), "output_t0")
    else:
        raise ValueError(f"bad output_style {cd.output_style}")
    add(1, "output_format")
    add([1] * int(cd.num_eqn), "iout_q")
    if cd.num_aux > 0:
        add([0] * int(cd.num_aux), "iout_aux")
        add(bool(cd.output_aux_onlyonce), "output_aux_onlyonce")
    add(float(cd.dt_initial), "dt_initial")
    add(float(cd.dt_max), "dt_max")
    add(float(cd.cfl_max), "cfl_max")
    add(float(cd.cfl_desired), "cfl_desired")
    add(int(cd.steps_max), "steps_max")
    add(bool(cd.dt_variable), "dt_variable")
    add(int(cd.order), "order")
    add(cd.transverse_code() if cd.num_dim > 1 else 0, "transverse_waves")
    add(cd.split_code() if cd.num_dim > 1 else 0, "dimensional_split")
    add(int(cd.verbosity), "verbosity")
    add(cd.source_code(), "source_split")
    add(int(cd.capa_index), "capa_index")
    add(bool(cd.use_fwaves), "use_fwaves")
    add(cd.limiter_codes(), "limiter")
    add(int(cd.num_ghost), "num_ghost")
    lo, hi = cd.bc_codes()
    add(lo, "bc_lower")
    add(hi, "bc_upper")
    add(bool(cd.restart), "restart")
    if cd.restart:
        add(int("".join(ch for ch in str(cd.restart_file) if ch.isdigit()) or 0), "restart_frame")
    with open(fname, "w") as f:
        f.write("# claw.data written by classic_b200.data\n\n")
        f.write("\n".join(lines) + "\n")


def _values(line):
    body = line.split("=:")[0].split()
    out = []
    for tok in body:
        t = tok.strip()
        if t in ("T", ".true.", "True"):
            out.append(True)
        elif t in ("F", ".false.", "False"):
            out.append(False)
        else:
            try:
                out.append(int(t))
            except ValueError:
                out.append(float(t.replace("d", "e").replace("D", "e")))
    return out


def read_claw_data(fname="claw.data") -> ClawInputData:
    """Parse claw.data (leading '#' comment lines skipped, as opendatafile
    does, src/2d/opendatafile.f:31-39) back into a ClawInputData."""
    with open(fname) as f:
        lines = [ln for ln in f if ln.strip() and not ln.lstrip().startswith("#")]
    it = iter(lines)
    nxt = lambda: _values(next(it))  # noqa: E731
    ndim = nxt()[0]
    cd = ClawInputData(ndim)
    cd.lower = [float(x) for x in nxt()]
    cd.upper = [float(x) for x in nxt()]
    cd.num_cells = [int(x) for x in nxt()]
    cd.num_eqn = nxt()[0]
    cd.num_waves = nxt()[0]
    cd.num_aux = nxt()[0]
    cd.t0 = float(nxt()[0])
    cd.output_style = nxt()[0]
    if cd.output_style == 1:
        cd.num_output_times = nxt()[0]
        cd.tfinal = float(nxt()[0])
        cd.output_t0 = bool(nxt()[0])
    elif cd.output_style == 2:
        n = nxt()[0]
        cd.output_times = [float(x) for x in nxt()][:n]
    else:
        cd.output_step_interval = nxt()[0]
        cd.total_steps = nxt()[0]
        cd.output_t0 = bool(nxt()[0])
    nxt()  # output_format
    nxt()  # iout_q
    if cd.num_aux > 0:
        nxt()
        cd.output_aux_onlyonce = bool(nxt()[0])
    cd.dt_initial = float(nxt()[0])
    cd.dt_max = float(nxt()[0])
    cd.cfl_max = float(nxt()[0])
    cd.cfl_desired = float(nxt()[0])
    cd.steps_max = nxt()[0]
    cd.dt_variable = bool(nxt()[0])
    cd.order = nxt()[0]
    cd.transverse_waves = nxt()[0]
    cd.dimensional_split = nxt()[0]
    cd.verbosity = nxt()[0]
    cd.source_split = nxt()[0]
    cd.capa_index = nxt()[0]
    cd.use_fwaves = bool(nxt()[0])
    cd.limiter = nxt()
    cd.num_waves = len(cd.limiter)
    cd.num_ghost = nxt()[0]
    cd.bc_lower = nxt()
    cd.bc_upper = nxt()
    try:
        cd.restart = bool(nxt()[0])
    except StopIteration:
        cd.restart = False
    return cd


def install_clawutil_alias():
    """Make ``from clawpack.clawutil import data`` resolve to this module so
    an unchanged setrun.py imports the shim."""
    this = sys.modules[__name__]
    if "clawpack" not in sys.modules:
        pkg = types.ModuleType("clawpack")
        pkg.__path__ = []
        sys.modules["clawpack"] = pkg
    if "clawpack.clawutil" not in sys.modules:
        sub = types.ModuleType("clawpack.clawutil")
        sub.__path__ = []
        sys.modules["clawpack.clawutil"] = sub
        sys.modules["clawpack"].clawutil = sub
    sys.modules["clawpack.clawutil"].data = this
    sys.modules["clawpack.clawutil.data"] = this
    return this
