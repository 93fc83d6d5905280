"""Record formats of the reference's text outputs (fribois2d_b200.io)."""
import numpy as np

from fribois2d_b200 import HIST_COLS, HIST_NAMES
from fribois2d_b200 import io as fio


def test_fortran_e16_9_known_answers():
    # gfortran prints Ew.d as [sign]0.<d digits>E<sign><2 digits>, right-justified
    assert fio.fortran_e(1.0) == " 0.100000000E+01"
    assert fio.fortran_e(-2.5e-3) == "-0.250000000E-02"
    assert fio.fortran_e(0.0) == " 0.000000000E+00"
    assert fio.fortran_e(123456789.0) == " 0.123456789E+09"
    assert fio.fortran_e(0.9999999999) == " 0.100000000E+01"       # rounds up into the next decade
    assert fio.fortran_e(1.0e-120) == " 0.100000000-119"            # three-digit exponent drops the E
    assert len(fio.fortran_e(-1.0e200)) == 16
    assert fio.fortran_i(7) == "    7" and fio.fortran_i(123456) == "*****"


def _hist(rows=3):
    h = np.zeros((rows, HIST_COLS))
    for i in range(rows):
        h[i] = np.arange(HIST_COLS) * 0.5 + i
    return h


def test_forcecomp_and_rbkin_records():
    h = _hist()
    fc = fio.forcecomp_lines(h)
    assert len(fc) == 3
    for ln in fc:   # eight e16.9 fields separated by 2x
        assert len(ln) == 8 * 16 + 7 * 2
        vals = [float(ln[i * 18:i * 18 + 16]) for i in range(8)]
        assert vals[0] == h[fc.index(ln), HIST_NAMES.index("time")]
    rb = fio.rbkin_lines(h)
    assert all(len(ln) == 10 * 16 + 9 * 2 for ln in rb)
    assert float(rb[1][:16]) == h[1, HIST_NAMES.index("time_end")]


def test_fluid_rep_record_has_integer_step():
    h = _hist(2)
    ln = fio.fluid_rep_lines(h, ns0=41)
    assert ln[0][18:23] == "   41" and ln[1][18:23] == "   42"
    assert len(ln[0]) == 16 + 2 + 5 + 5 * (2 + 16)


def test_reporter_appends(tmp_path):
    r = fio.Reporter(str(tmp_path))
    r.write(_hist(2), 0)
    r.write(_hist(3), 2)
    for name, n in (("forcecomp.out", 5), ("rbkin.out", 5), ("fluid_rep.out", 5)):
        assert len((tmp_path / name).read_text().splitlines()) == n


def test_master_rigid_text_round_trips():
    t = fio.master_rigid_text(1.25, 1e-3, 1e-3, [0.1, 0.2, 0.3], [1, 2, 3], [-1e-9, 0, 5])
    lines = t.splitlines()
    assert len(lines) == 5
    assert float(lines[0]) == 1.25
    assert [float(x) for x in lines[2].split()] == [0.1, 0.2, 0.3]
