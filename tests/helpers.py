"""Shared helpers for the parity tests (oracle = the CPU restatement)."""
import numpy as np


def e26(q):
    """Round to the 16 significant digits Fortran e26.16 writes."""
    f = np.vectorize(lambda v: float(f"{v:.15e}"))
    return f(np.asarray(q, dtype=np.float64))


def frame_sum(field):
    """Sum of one field as the reference's regression check forms it: pyclaw
    stores a frame as q[m, i, j(, k)] (x index slowest in C order), so numpy
    sums the interior with the last axis fastest.  `field` is the SoA
    [(mz,)(my,)mx] layout used here."""
    a = e26(field)
    return float(np.ascontiguousarray(a.transpose(tuple(range(a.ndim))[::-1])).sum())


def rel_diff(a, b):
    """Normwise relative difference per field: max|a-b| / max|b|."""
    a = np.asarray(a)
    b = np.asarray(b)
    out = []
    for m in range(a.shape[0]):
        den = np.max(np.abs(b[m]))
        num = np.max(np.abs(a[m] - b[m]))
        out.append(num / den if den > 0 else num)
    return np.array(out)


def same(a, b):
    """Bit-for-bit value equality (+0 == -0); a NaN matches only a NaN at the
    same position (the Roe solver can leave a strong rarefaction with
    negative pressure, on either side identically)."""
    return bool(np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True))
