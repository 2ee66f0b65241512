"""Host helpers of the time-to-L1 study (classic_b200/accuracy.py)."""
import numpy as np

from classic_b200 import accuracy


def test_block_average_and_norms_host():
    q = np.arange(2 * 4 * 4, dtype=np.float64).reshape(2, 4, 4)
    b = accuracy.block_average(q, 2)
    assert b.shape == (2, 2, 2)
    assert b[0, 0, 0] == np.mean([0, 1, 4, 5])
    assert accuracy.l1_norms(b, b + 1.0, 0.5, 0.25) == [0.5, 0.5]
