"""The INT8 digit-slice product restated in NumPy (oracle/i8x8.py): the
digits reconstruct the operands, the integer class sums stay inside int32,
and the product is as accurate as FP64 (error against an extended-precision
product, normalised by sum_k |a_ik| |b_jk|)."""
import numpy as np
import pytest

from oracle import i8x8


def test_digits_reconstruct_rows():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((40, 300)) * np.exp(rng.uniform(-20, 20, (40, 1)))
    X[3] = 0.0
    e, D = i8x8.digits(X)
    assert all(np.abs(d).max() <= 127 for d in D)
    back = sum(d.astype(np.float64) * np.ldexp(1.0, -7 * (i + 1)) for i, d in enumerate(D))
    back = back * np.ldexp(1.0, e)[:, None]
    mu = np.abs(X).max(axis=1, keepdims=True)
    assert np.all(np.abs(back - X) <= np.ldexp(1.0, -55) * np.maximum(mu, 1e-300))
    assert np.all(back[3] == 0.0)


@pytest.mark.parametrize("K", [77, 1024, 2048])
def test_class_sums_fit_int32(K):
    # worst case: every digit +-127; class t sums t + 1 products of K terms
    assert i8x8.S * K * 127 * 127 < 2 ** 31


@pytest.mark.parametrize("M,N,K", [(64, 48, 1024), (40, 30, 77)])
def test_product_is_fp64_accurate(M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = rng.standard_normal((M, K)) * np.exp(rng.uniform(-3, 3, (M, 1)))
    B = rng.standard_normal((N, K)) * np.exp(rng.uniform(-3, 3, (N, 1)))
    C = i8x8.gemm(A, B)
    ref = A.astype(np.longdouble) @ B.T.astype(np.longdouble)
    scale = np.abs(A) @ np.abs(B).T
    err = float(np.max(np.abs(C - ref) / scale))
    dgemm = float(np.max(np.abs(A @ B.T - ref) / scale))
    assert err <= max(5e-16, 2.0 * dgemm), (err, dgemm)
    # fewer digits are measurably worse: the eighth one is needed
    assert float(np.max(np.abs(i8x8.gemm(A, B, s=7) - ref) / scale)) > 10 * err
