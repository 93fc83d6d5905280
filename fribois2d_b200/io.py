"""Text output in the reference's record formats.

Each writer takes the per-step history rows that `Solver.advance` returns
(columns HIST_NAMES) and appends lines formatted exactly as the reference's
FORMAT statements print them:

* forcecomp.out -- rigid.F90:431-433, format 933: time, Fy, Fz, M, Fyp, Fzp,
  Fyv, Fzv, each e16.9, separated by 2x;
* rbkin.out     -- ttime.F90:146-149, format 932: time, cmp_np1(3),
  cmv_np1(3), cma_np1(3);
* fluid_rep.out -- ttime.F90:142-144, format 931: time, ns (i5), dt, cflm,
  dmax, ektot, vorti (the diagnostics columns of the history rows).

Fortran Ew.d output is restated here: a sign position (blank for
non-negative values), "0.", d significant digits rounded to nearest, and a
four-character exponent field "E+ee" (or "+eee" when |exponent| > 99, the
letter dropped as the standard prescribes).  A format's trailing 2x before
an unused edit descriptor moves the position only, so no trailing blanks are
written.
"""
from __future__ import annotations

import math
import os
from typing import Iterable, Sequence

import numpy as np

from . import HIST_NAMES


def fortran_e(x: float, w: int = 16, d: int = 9) -> str:
    """One value in Fortran Ew.d editing (gfortran layout, 0.ddd form)."""
    x = float(x)
    if math.isnan(x):
        return "NaN".rjust(w)
    if math.isinf(x):
        return ("-Infinity" if x < 0 else "Infinity").rjust(w)
    sign = "-" if (x < 0 or (x == 0.0 and math.copysign(1.0, x) < 0)) else " "
    a = abs(x)
    if a == 0.0:
        mant, exp = "0" * d, 0
    else:
        s = f"{a:.{d - 1}e}"            # d.ddd...e+XX: d significant digits, rounded
        m, e = s.split("e")
        mant = m.replace(".", "")
        exp = int(e) + 1                 # 0.ddd form
    if abs(exp) <= 99:
        es = f"E{'+' if exp >= 0 else '-'}{abs(exp):02d}"
    else:
        es = f"{'+' if exp >= 0 else '-'}{abs(exp):03d}"
    body = f"0.{mant}{es}"
    out = (sign if sign == "-" else " ") + body
    if len(out) > w:                     # no room for the sign blank / leading zero
        out = (sign.strip() + "." + mant + es)
    return out.rjust(w) if len(out) <= w else "*" * w


def fortran_i(n: int, w: int = 5) -> str:
    s = str(int(n))
    return s.rjust(w) if len(s) <= w else "*" * w


def _col(name: str) -> int:
    return HIST_NAMES.index(name)


def forcecomp_lines(hist: np.ndarray) -> list:
    """format 933 (rigid.F90:432): time, forcm(2), momcm, fyp, fzp, fyv, fzv."""
    cols = [_col(c) for c in ("time", "Fy", "Fz", "M", "Fyp", "Fzp", "Fyv", "Fzv")]
    return ["  ".join(fortran_e(row[c]) for c in cols) for row in np.atleast_2d(hist)]


def rbkin_lines(hist: np.ndarray) -> list:
    """format 932 (ttime.F90:146): time (end of step), cmp_np1, cmv_np1, cma_np1."""
    cols = [_col(c) for c in ("time_end", "py", "pz", "pa", "vy", "vz", "va", "ay", "az", "aa")]
    return ["  ".join(fortran_e(row[c]) for c in cols) for row in np.atleast_2d(hist)]


def fluid_rep_lines(hist: np.ndarray, ns0: int) -> list:
    """format 931 (ttime.F90:142): time, ns, dt, cflm, dmax, ektot, vorti."""
    out = []
    for i, row in enumerate(np.atleast_2d(hist)):
        vals = [fortran_e(row[_col("time_end")]), fortran_i(ns0 + i), fortran_e(row[_col("dt")]),
                fortran_e(row[_col("cflm_end")]), fortran_e(row[_col("dmax")]),
                fortran_e(row[_col("ektot")]), fortran_e(row[_col("vorti")])]
        out.append("  ".join(vals))
    return out


def append(path: str, lines: Iterable[str]) -> None:
    with open(path, "a") as f:
        for ln in lines:
            f.write(ln + "\n")


class Reporter:
    """Appends the reference's three per-step report files under outdir."""

    def __init__(self, outdir: str):
        os.makedirs(outdir, exist_ok=True)
        self.outdir = outdir

    def write(self, hist: np.ndarray, ns0: int) -> None:
        append(os.path.join(self.outdir, "forcecomp.out"), forcecomp_lines(hist))
        append(os.path.join(self.outdir, "rbkin.out"), rbkin_lines(hist))
        append(os.path.join(self.outdir, "fluid_rep.out"), fluid_rep_lines(hist, ns0))


def master_rigid_text(time: float, dt: float, dt_o: float, cmp: Sequence[float], cmv: Sequence[float],
                      cma: Sequence[float]) -> str:
    """restart/master_rigid.dat as ttime.F90:117-124 writes it with list-directed
    output (gfortran: reals as 17 significant digits in fields of 25)."""
    def ld(vals):
        return "".join(f"{float(v):25.17g}".replace("e", "E") for v in vals) + "\n"
    return ld([time]) + ld([dt, dt_o]) + ld(cmp) + ld(cmv) + ld(cma)
