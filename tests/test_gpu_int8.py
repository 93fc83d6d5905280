"""FP64 eigen transforms on the INT8 tensor cores (FB_POISSON_INT8X8).

Every row of each operand is scaled by a power of two and cut into 8 signed
8-bit digits; the digit products are exact int32 sums on the tensor cores
and are added in FP64.  Tolerances: the GEMM against an extended-precision
product, normalised by sum_k |a_ik| |b_jk| (the scale of FP64 rounding in any
summation order): the dropped digit pairs and the FP64 additions stay within
twice an FP64 DGEMM's error in the same check (5e-16 of it at most).  The time step
against the plain FP64 path: two FP64-accurate transforms that differ only
in rounding, 1e-12 relative per step.
"""
import numpy as np
import pytest

import fribois2d_b200 as fb
from fribois2d_b200 import case as cases
from paritylib import rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(96, 80, 1000), (130, 70, 200), (256, 192, 1024), (200, 130, 77)])
def test_i8x8_gemm_is_fp64_accurate(M, N, K):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    # rows of very different magnitude: the per-row power-of-two scaling
    A = rng.standard_normal((M, K)) * np.exp(rng.uniform(-3, 3, (M, 1)))
    B = rng.standard_normal((N, K)) * np.exp(rng.uniform(-3, 3, (N, 1)))
    C = fb.gemm_i8x8(A, B)
    ref = A.astype(np.longdouble) @ B.T.astype(np.longdouble)
    scale = np.abs(A) @ np.abs(B).T
    err = float(np.max(np.abs(C - ref) / scale))
    dgemm = float(np.max(np.abs(A @ B.T - ref) / scale))
    print(f"i8x8 {err:.3e}  fp64 {dgemm:.3e}")
    # as accurate as an FP64 product: within the FP64 rounding scale, and
    # never more than twice the error of numpy's FP64 product
    assert err <= max(5e-16, 2.0 * dgemm), (err, dgemm)


def test_i8x8_gemm_zero_rows():
    """An all-zero row or column gives an exact zero row or column."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((64, 300))
    B = rng.standard_normal((40, 300))
    A[5] = 0.0
    B[7] = 0.0
    C = fb.gemm_i8x8(A, B)
    assert np.all(C[5] == 0.0) and np.all(C[:, 7] == 0.0)
    assert float(np.max(np.abs(C - A @ B.T))) <= 1e-12


def _run(c, path, mode, steps):
    s = fb.Solver(path)
    s.set_poisson(mode)
    q2 = s.get("q2")
    q2[1:c.n3m + 1] += c.v_perturbation()
    s.set("q2", q2)
    h = s.advance(0, steps)
    out = {f: s.get(f) for f in ("q2", "q3", "pr")}
    s.close()
    return out, h


@pytest.mark.parametrize("maker,steps", [(cases.tiny_rectangle, 20), (cases.viv_cylinder_384x256, 10)])
def test_int8_step_matches_fp64(maker, steps, tmp_path):
    c = maker()
    path = c.write(str(tmp_path / c.name))
    a, ha = _run(c, path, fb.POISSON_FP64, steps)
    b, hb = _run(c, path, fb.POISSON_INT8X8, steps)
    n2m, n3m = c.n2m, c.n3m
    for f in ("q2", "q3", "pr"):
        e = rel(b[f][1:n3m + 1, :n2m], a[f][1:n3m + 1, :n2m])
        print(f, e)
        assert e <= 1e-12 * steps, (f, e)
    for col in (1, 2, 3, 9, 10, 11):   # forces and displacements
        rng_ = max(np.ptp(ha[:, col]), np.max(np.abs(ha[:, col])), 1e-30)
        assert np.max(np.abs(hb[:, col] - ha[:, col])) <= 1e-10 * rng_, col


def test_i8x8_gemm_equals_restatement():
    """The device computes exactly the NumPy restatement's operations: the
    digits, the exact integer class sums and the FP64 additions in the same
    order give the same bits."""
    from oracle import i8x8
    rng = np.random.default_rng(11)
    A = rng.standard_normal((100, 300)) * np.exp(rng.uniform(-5, 5, (100, 1)))
    B = rng.standard_normal((70, 300)) * np.exp(rng.uniform(-5, 5, (70, 1)))
    B[9] = 0.0
    np.testing.assert_array_equal(fb.gemm_i8x8(A, B), i8x8.gemm(A, B))


def test_int8_tile_widths_agree_bitwise(tmp_path, monkeypatch):
    """The digit products are exact integer sums added in FP64 in a fixed
    order, so the product tile width (128 x 64, 128 x 48 or 128 x 32, chosen
    per grid size by the autotuner) cannot change a bit of the result."""
    c = cases.viv_cylinder_384x256()
    path = c.write(str(tmp_path / c.name))
    out = []
    for width in ("64", "48", "32"):
        monkeypatch.setenv("FRIBOIS2D_I8_TILE", width)
        a, h = _run(c, path, fb.POISSON_INT8X8, 5)
        out.append((a, h))
    (a, ha) = out[0]
    for b, hb in out[1:]:
        for f in ("q2", "q3", "pr"):
            np.testing.assert_array_equal(a[f], b[f], err_msg=f)
        np.testing.assert_array_equal(ha, hb)
