"""The ClawRunData drop-in: string codes, claw.data round trip, and the
reference examples' unchanged setrun.py files (when the environment variable
CLAW_CLASSIC_EXAMPLES names the examples/ directory of a clawpack/classic
checkout; skipped otherwise)."""
import importlib.util
import os

import numpy as np
import pytest

from classic_b200 import data
from classic_b200.solver import make_config

REF = os.environ.get("CLAW_CLASSIC_EXAMPLES", "")


def test_codes_and_config():
    rd = data.ClawRunData("classic", 2)
    cd = rd.clawdata
    cd.limiter = ["mc", "vanleer"]
    cd.num_waves = 2
    cd.bc_lower = ["wall", "periodic"]
    cd.bc_upper = ["extrap", "periodic"]
    cd.transverse_waves = "all"
    cfg = make_config(cd, "acoustics_2d", {"rho": 1.0, "bulk": 4.0})
    assert list(cfg.limiter)[:2] == [4, 3]
    assert list(cfg.bc_lower)[:2] == [3, 2] and list(cfg.bc_upper)[:2] == [1, 2]
    assert cfg.transverse_waves == 2 and cfg.solver_id == 1
    with pytest.raises(ValueError):
        cd.limiter = ["nope", "mc"]
        make_config(cd, "acoustics_2d", {"rho": 1.0, "bulk": 4.0})


def test_claw_data_round_trip(tmp_path):
    rd = data.ClawRunData("classic", 2)
    cd = rd.clawdata
    cd.num_cells = [40, 120]
    cd.lower, cd.upper = [0.2, 0.0], [1.0, 6.283185307179586]
    cd.num_aux, cd.capa_index = 3, 3
    cd.limiter, cd.num_waves = ["vanleer"], 1
    cd.bc_lower, cd.bc_upper = ["extrap", "periodic"], ["extrap", "periodic"]
    p = rd.new_UserData("probdata", "setprob.data")
    p.add_param("A1", 1.0, "amplitude")
    rd.write(str(tmp_path))
    back = data.read_claw_data(str(tmp_path / "claw.data"))
    assert back.num_cells == [40, 120]
    assert back.lower == [0.2, 0.0] and back.upper[1] == 6.283185307179586
    assert back.limiter == [3] and back.bc_lower == [1, 2] and back.bc_upper == [1, 2]
    assert back.capa_index == 3 and back.num_aux == 3
    assert "A1" in (tmp_path / "setprob.data").read_text()


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="CLAW_CLASSIC_EXAMPLES not set")
@pytest.mark.parametrize("example", ["acoustics_1d_example1", "acoustics_1d_heterogeneous",
                                     "acoustics_2d_radial", "advection_2d_annulus",
                                     "acoustics_3d_heterogeneous", "advection_1d_example1",
                                     "euler_1d_wcblast"])
def test_reference_setrun_runs_unchanged(example, tmp_path):
    data.install_clawutil_alias()
    path = os.path.join(REF, example, "setrun.py")
    spec = importlib.util.spec_from_file_location(f"setrun_{example}", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    rd = mod.setrun("classic")
    rd.write(str(tmp_path))
    back = data.read_claw_data(str(tmp_path / "claw.data"))
    assert back.num_cells == list(rd.clawdata.num_cells)
    assert back.limiter == rd.clawdata.limiter_codes()


def _cfg_fields(cfg):
    out = {}
    for name, _ in cfg._fields_:
        v = getattr(cfg, name)
        out[name] = list(v) if hasattr(v, "__len__") else v
    return out


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="CLAW_CLASSIC_EXAMPLES not set")
@pytest.mark.parametrize("example,solver,params", [
    ("advection_1d_example1", "advection_1d", {"u": 1.0}),
    ("euler_1d_wcblast", "euler_roe_1d", {"gamma": 1.4}),
])
def test_builtin_problem_matches_reference_setrun(example, solver, params):
    """The problem builders restate the examples' setrun.py: the unchanged
    setrun.py and the builder give the same claw_config."""
    from classic_b200 import problems
    data.install_clawutil_alias()
    path = os.path.join(REF, example, "setrun.py")
    spec = importlib.util.spec_from_file_location(f"setrun_{example}_cfg", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    ref = _cfg_fields(make_config(mod.setrun("classic").clawdata, solver, params))
    rd, s, p, _, _ = getattr(problems, example)()
    assert s == solver and p == params
    ours = _cfg_fields(make_config(rd.clawdata, s, p))
    assert ours == ref
