"""The device-wait failure path of the 2D step kernels.

Every TMA/mbarrier wait in the step kernels is bounded: when a wait runs out
the kernel drains its own copies, raises an error flag in the control block
and returns, so the GPU never hangs.  The test hook claw_debug_fault makes the
warps of strip 0 skip the copy of one row and shortens the wait limit to 2 ms:
the wait on that row then runs out and nothing faults (no copy is in flight
to the skipped slot).  The step whose wait ran out is not accepted:
claw_advance and claw_step return CLAW_E_DEVICE, the handle keeps the q of the
last accepted step, and once the hook is off the next call runs normally and
matches an undisturbed handle bit for bit.  Analogue in the reference: the
error returns of claw2 (src/2d/claw2.f:288-310) leave q as it was."""
import ctypes

import numpy as np
import pytest

from classic_b200 import _lib, problems
from classic_b200.solver import Solver

pytestmark = pytest.mark.gpu

CLAW_E_DEVICE = -4
CTL_ERR_TMA_TIMEOUT = 1


@pytest.mark.parametrize("precision", ["fp64", "fp64_fma"])
@pytest.mark.parametrize("skip_row", [5, -2])
def test_wait_timeout_reported_and_state_kept(precision, skip_row):
    rd, solver, params, q0, _ = problems.radial_acoustics_2d(n=128)
    s = Solver(rd.clawdata, solver, params, precision=precision)
    ref = Solver(rd.clawdata, solver, params, precision=precision)
    try:
        s.set_q(q0)
        ref.set_q(q0)
        info, st = s.advance(0.0, 0.05, 0.01)
        info_r, st_r = ref.advance(0.0, 0.05, 0.01)
        assert info == 0 and info_r == 0
        q1 = s.get_q()
        lib = _lib.load()

        assert lib.claw_debug_fault(s._h, 2_000_000, skip_row) == 0
        stats = _lib.ClawStats()
        rc = lib.claw_advance(s._h, 0.05, 0.1, st["dt_next"], ctypes.byref(stats))
        assert rc == CLAW_E_DEVICE, lib.claw_last_error().decode()
        assert stats.device_error & CTL_ERR_TMA_TIMEOUT
        assert stats.steps_taken == 0
        assert np.array_equal(s.get_q(), q1)
        cfl = ctypes.c_double(0.0)
        rc = lib.claw_step(s._h, st["dt_next"], ctypes.byref(cfl))
        assert rc == CLAW_E_DEVICE
        assert np.array_equal(s.get_q(), q1)

        # hook off: the handle works again and equals the undisturbed one
        assert lib.claw_debug_fault(s._h, 0, -3) == 0
        info, st2 = s.advance(0.05, 0.1, st["dt_next"])
        info_r, st_r2 = ref.advance(0.05, 0.1, st_r["dt_next"])
        assert info == 0 and info_r == 0
        assert st2["steps_taken"] == st_r2["steps_taken"]
        assert np.array_equal(s.get_q(), ref.get_q())
    finally:
        s.close()
        ref.close()
