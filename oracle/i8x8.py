"""Test infrastructure: a NumPy restatement of the INT8 digit-slice product
of fribois2d_b200/csrc/tc_gemm.cu (k_i8_rowmax, k_i8_digits, k_i8x8_gemm),
used to check the device result bit for bit and the method's error bound.

The method is the Ozaki scheme (Ozaki, Ogita, Oishi and Rump, "Error-free
transformations of matrix multiplication by using fast routines of matrix
multiplication and its applications", Numer. Algorithms 59, 2012) in its
integer form with power-of-two row scaling: every row of A (and of B) is
scaled by 2^-e with |a| < 2^e and cut into S signed digits of 7 bits,
a = sum_i d_i 128^-(i+1); C = A B^T is then
    C(r, c) = 2^(e(r) + f(c)) sum_t 128^-(t+2) G_t(r, c),
    G_t = sum_{i+j=t} D_i E_j^T   (exact integer products, t < S),
the G_t added in FP64 from t = S-1 down to 0, then the two power-of-two
scales applied.
"""
from __future__ import annotations

import numpy as np

S = 8


def digits(X: np.ndarray, s: int = S):
    """Row exponents e (|X[r]| < 2^e[r]; 0 for a zero row) and the s digit
    planes of X (int64 arrays of X's shape)."""
    X = np.asarray(X, dtype=np.float64)
    mu = np.abs(X).max(axis=1)
    _, e = np.frexp(mu)                      # mu = m 2^e, 0.5 <= m < 1 (e = 0 for mu = 0)
    e = np.where(mu > 0, e, 0).astype(np.int64)
    a = X * np.ldexp(1.0, -e)[:, None]
    out = []
    for _ in range(s):
        a = a * 128.0
        d = np.trunc(a)
        a = a - d
        out.append(d.astype(np.int64))
    return e, out


def gemm(A: np.ndarray, B: np.ndarray, s: int = S) -> np.ndarray:
    """C = A @ B.T as the device computes it (same operations, same order)."""
    ea, Da = digits(A, s)
    eb, Db = digits(B, s)
    acc = np.zeros((A.shape[0], B.shape[0]), dtype=np.float64)
    for t in range(s - 1, -1, -1):
        G = sum(Da[i] @ Db[t - i].T for i in range(t + 1))
        acc = acc + G.astype(np.float64) * np.ldexp(1.0, -7 * (t + 2))
    return (acc * np.ldexp(1.0, ea)[:, None]) * np.ldexp(1.0, eb)[None, :]
