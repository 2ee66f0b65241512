"""classic_b200 — B200-native Clawpack Classic wave-propagation step.

Python host layer over the sm_100a CUDA library (include/claw_b200.h):

* ``data``      — ClawRunData drop-in (setrun.py interface, claw.data I/O)
* ``solver``    — ``Solver`` (one grid on the GPU) and ``run`` (claw2ez loop)
* ``frames``    — fort.qNNNN / fort.tNNNN frame files (out2 format)
* ``problems``  — the reference examples and the synthetic workloads
"""
from .data import ClawRunData, install_clawutil_alias  # noqa: F401
from .solver import Solver, run, make_config  # noqa: F401

__all__ = ["ClawRunData", "Solver", "run", "make_config", "install_clawutil_alias"]
