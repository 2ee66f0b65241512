"""fort.q / fort.t frame files (src/2d/out2.f, src/1d/out1.f, src/3d/out3.f
layout) and the claw2ez restart path, on the host."""
import os

import numpy as np
import pytest

from classic_b200 import frames, problems


def test_fortran_e_edit_descriptor():
    assert frames.fortran_e(1.0) == "    0.1000000000000000E+01"
    assert frames.fortran_e(-2.5e-3) == "   -0.2500000000000000E-02"
    assert frames.fortran_e(0.0) == "    0.0000000000000000E+00"
    assert frames.fortran_e(1e-120).strip() == "0.1000000000000000-119"
    assert len(frames.fortran_e(123.456)) == 26


@pytest.mark.parametrize("shape", [(2, 17), (3, 5, 7), (4, 3, 4, 5)])
def test_write_read_roundtrip(tmp_path, shape):
    rng = np.random.default_rng(len(shape))
    q = rng.standard_normal(shape)
    q.flat[0] = 1e-120  # flushed to zero as out2 does
    nd = len(shape) - 1
    frames.write_frame(str(tmp_path), 3, 0.25, q, [-1.0] * nd, [0.1] * nd, maux=0, nghost=2)
    t, r = frames.read_frame(str(tmp_path), 3)
    assert t == 0.25
    assert r.shape == q.shape
    expect = np.vectorize(lambda v: float(f"{v:.15e}"))(q)
    expect.flat[0] = 0.0
    assert np.array_equal(r, expect)


def test_2d_layout_matches_out2(tmp_path):
    q = np.arange(2 * 2 * 3, dtype=float).reshape(2, 2, 3) + 1.0
    fq, ft = frames.write_frame(str(tmp_path), 1, 0.5, q, [0.0, -1.0], [0.5, 0.25])
    lines = open(fq).read().split("\n")
    assert lines[0] == "    1                 grid_number"
    assert lines[1] == "    1                 AMR_level"
    assert lines[2] == "    3                 mx"
    assert lines[3] == "    2                 my"
    assert lines[4].endswith("    xlow") and len(lines[4]) == 26 + 8
    assert lines[8] == ""
    # first row: cells (i=1..3, j=1), equation index fastest on a line
    assert lines[9] == frames.fortran_e(1.0) + frames.fortran_e(7.0)
    assert lines[12].strip() == ""
    tl = open(ft).read().split("\n")
    assert tl[0] == frames.fortran_e(0.5) + "    time"
    assert tl[1] == "    2                 meqn"
    assert tl[4] == "    2                 ndim"


def test_fort_info_records(tmp_path):
    """fort.info: claw2ez's format 1010 record (src/2d/claw2ez.f:308-309,
    319-322) per output frame, D15.4 reals, I5 info, I4 step count (asterisks
    when it does not fit); start_info truncates the file as the OPEN at the
    start of a run does."""
    out = str(tmp_path)
    path = frames.start_info(out)
    with open(path, "a") as f:
        f.write("stale\n")
    frames.start_info(out)
    st = {"dt_min": 1.25e-3, "dt_max_taken": 2.5e-3, "dt_next": 2.4e-3,
          "cfl_max_seen": 0.9, "cfl_last": 0.8999, "steps_taken": 40}
    frames.append_info(out, 0.1, 0, st)
    frames.append_info(out, 0.2, 11, dict(st, steps_taken=12345, dt_min=-0.0))
    text = open(path).read()
    assert text == (
        "tend =     0.1000D+00\n"
        "info =    0\n"
        "smallest dt =     0.1250D-02\n"
        "largest dt =     0.2500D-02\n"
        "last dt =     0.2400D-02\n"
        "largest cfl =     0.9000D+00\n"
        "last cfl =     0.8999D+00\n"
        "steps taken =  40\n"
        "\n"
        "tend =     0.2000D+00\n"
        "info =   11\n"
        "smallest dt =    -0.0000D+00\n"
        "largest dt =     0.2500D-02\n"
        "last dt =     0.2400D-02\n"
        "largest cfl =     0.9000D+00\n"
        "last cfl =     0.8999D+00\n"
        "steps taken =****\n"
        "\n")
