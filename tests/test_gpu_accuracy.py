"""Time to an L1 error on the 2D radial acoustics workload (the metric's
second half: plain FP64 against the FP32 and contracted builds), at reduced
sizes: 128^2 and 256^2 against a 512^2 truth, to t = 0.3.

Properties that hold at every size:
  * the error falls as the grid is refined (by more than 1.5x per doubling
    for this smooth pulse with MC);
  * the contracted FP64 build has the reference order's L1 to 1e-9 relative
    and takes the same steps;
  * FP32 has it to 1e-4 relative: rounding is far below the discretisation
    error, so the FP32 run reaches the same error in less time."""
import numpy as np
import pytest

from classic_b200 import accuracy

pytestmark = pytest.mark.gpu


def test_radial_time_to_l1_small():
    res = accuracy.radial_time_to_l1(sizes=(128, 256), truth_n=512, tfinal=0.3)
    rows = {(r["n"], r["precision"]): r for r in res["rows"]}
    for n in (128, 256):
        ref = rows[(n, "fp64")]
        assert ref["l1_p"] > 0 and np.isfinite(ref["l1_p"])
        assert rows[(n, "fp64_fma")]["steps"] == ref["steps"]
        assert abs(rows[(n, "fp64_fma")]["l1_p"] - ref["l1_p"]) <= 1e-9 * ref["l1_p"]
        assert abs(rows[(n, "fp32")]["l1_p"] - ref["l1_p"]) <= 1e-4 * ref["l1_p"]
    assert rows[(128, "fp64")]["l1_p"] > 1.5 * rows[(256, "fp64")]["l1_p"]


def test_ensemble_batched_equals_serial_and_is_faster():
    """Eight instances of the batched Euler workload: the batch reproduces one
    claw2 call per instance bit for bit (reference order) in less time."""
    res = accuracy.ensemble_batched_vs_serial(count=8)
    assert res["identical"], res["max_abs_diff"]
    assert res["batched"]["wall_ms"] < res["serial"]["wall_ms"]
