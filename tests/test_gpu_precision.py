"""Precision form of the Poisson solve: the 3xTF32 tcgen05 GEMM and the time
step that uses it (TF32 split transforms, FP64 tridiagonal solves, one FP64
refinement sweep on the Poisson residual).

Tolerances: the GEMM is checked element by element against FP64 products,
normalised by sum_k |a_ik| |b_jk| (the scale of the rounding of any
summation order): 3xTF32 keeps about 22 bits of each operand and
accumulates in FP32, so 1e-5 bounds it with margin.  The time step is
compared with the plain FP64 path: after the refinement sweep the projected
velocity agrees to 1e-9 relative per step, and lift and displacement
histories to 1e-6 of their range.
"""
import numpy as np
import pytest

import fribois2d_b200 as fb
from fribois2d_b200 import case as cases
from paritylib import rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bn", [64, 128, 1128, 1192, 1256])
@pytest.mark.parametrize("M,N,K", [(128, 128, 32), (200, 130, 77), (256, 384, 1000), (768, 1024, 1024)])
def test_tf32x3_gemm_matches_fp64(M, N, K, bn):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((N, K))
    C = fb.gemm_tf32x3(A, B, bn=bn)
    ref = A @ B.T
    scale = np.abs(A) @ np.abs(B).T
    err = np.max(np.abs(C - ref) / scale)
    assert err <= 1e-5, err
    # the split products really are used: a single TF32 product is an order
    # of magnitude or more further off (FP32 accumulation bounds both)
    one = _tf32(A) @ _tf32(B).T
    assert err <= 0.1 * np.max(np.abs(one - ref) / scale)


def _tf32(x):
    """Round to TF32 (10 explicit mantissa bits, nearest, ties away)."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = ((b + 0x1000) & 0xFFFFE000).astype(np.uint32)
    return b.view(np.float32).astype(np.float64)


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
def test_precision_step_matches_fp64(maker, steps, tmp_path):
    c = maker()
    path = c.write(str(tmp_path / c.name))
    a, ha = _run(c, path, fb.POISSON_FP64, steps)
    b, hb = _run(c, path, fb.POISSON_TF32X3, steps)
    n2m, n3m = c.n2m, c.n3m
    for f in ("q2", "q3"):
        e = rel(b[f][1:n3m + 1, :n2m], a[f][1:n3m + 1, :n2m])
        assert e <= 1e-9 * steps, (f, e)
    for col in (1, 2, 3, 9, 10, 11):   # forces and displacements
        rng_ = max(np.ptp(ha[:, col]), np.max(np.abs(ha[:, col])), 1e-30)
        assert np.max(np.abs(hb[:, col] - ha[:, col])) <= 1e-6 * rng_, col


def test_autotune_keeps_state_and_results(tmp_path):
    """Tuning times candidates on the live context: the state afterwards and
    the following steps are those of an untuned run (to round-off of the
    chosen tile shapes, which do not change the arithmetic)."""
    c = cases.tiny_rectangle()
    path = c.write(str(tmp_path / c.name))
    a, ha = _run(c, path, fb.POISSON_TF32X3, 5)
    s = fb.Solver(path)
    s.set_poisson(fb.POISSON_TF32X3)
    q2 = s.get("q2")
    q2[1:c.n3m + 1] += c.v_perturbation()
    s.set("q2", q2)
    tk, bn = s.autotune()
    assert tk in (32, 64) and bn in (64, 128, 1128, 1192, 1256)
    hb = s.advance(0, 5)
    for f in ("q2", "q3"):
        assert np.array_equal(s.get(f), a[f]), f
    assert np.array_equal(ha, hb)
    s.close()
