"""CPU model of the split-precision product (test infrastructure only).

The reference has no split-precision path (it calls DGEMM,
imcom_matrix.f90:699, and DGEMV, imcom_matrix.f90:734); this module restates
the library's own int8 digit-slice product so the tests can check the
tensor-core kernel bit for bit:

* operand row r is scaled by sigma_r = 2^(ilogb(max_k |x_rk|) + 2);
* N = rint(x / sigma * 2^(7 + 8(S-1))) is split into S balanced base-256
  digits, d_0 most significant (weight 2^-7), d_k weight 2^(-7-8k);
* D_t = sum_{k+l=t} d_k(A) d_l(B)^T for t < S is exact integer arithmetic
  (float64 matmul of integers whose partial sums stay below 2^53);
* acc = D_{S-1}; acc = acc * 2^-8 + D_t for t = S-2 .. 0 (each step one
  IEEE rounding, as the kernel does), then C = (alpha sigma_A 2^-14 sigma_B) acc
  (a power of two: exact).

Only ``tests/`` imports this module.
"""
from __future__ import annotations

import numpy as np


def row_scales(X: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Power-of-two scale per row of X (rows = operand rows) and the exponent
    e (scale = 2^e); zero rows get scale 0 (their digits are zero)."""
    mx = np.max(np.abs(X), axis=1)
    live = mx > 0
    e = np.zeros(X.shape[0], dtype=np.int64)
    _, ex = np.frexp(mx[live])          # mx = f 2^ex, f in [0.5, 1): ilogb = ex - 1
    e[live] = ex.astype(np.int64) - 1 + 2
    scale = np.where(live, np.ldexp(1.0, e), 0.0)
    return scale, e


def digits(X: np.ndarray, S: int) -> tuple[list[np.ndarray], np.ndarray]:
    """S digit planes (float64 holding integers) of the rows of X and the
    row scales."""
    X = np.asarray(X, dtype=np.float64)
    scale, e = row_scales(X)
    q = np.ldexp(X, -e[:, None])
    N = np.rint(np.ldexp(q, 7 + 8 * (S - 1))).astype(np.int64)
    planes = [None] * S
    for s in range(S - 1, 0, -1):
        d = ((N + 128) & 255) - 128
        planes[s] = d
        N = (N - d) >> 8
    planes[0] = N
    assert np.all(np.abs(planes[0]) <= 65)
    return [p.astype(np.float64) for p in planes], scale


def split_product(Arows: np.ndarray, Brows: np.ndarray, S: int, alpha: float = 1.0):
    """C = alpha * Arows @ Brows.T (M x N) as the split product computes it."""
    da, sa = digits(Arows, S)
    db, sb = digits(Brows, S)
    acc = None
    for t in range(S - 1, -1, -1):
        D = np.zeros((Arows.shape[0], Brows.shape[0]))
        for k in range(t + 1):
            D += da[k] @ db[t - k].T
        assert np.max(np.abs(D)) < 2.0 ** 31
        acc = D if acc is None else acc * 2.0 ** -8 + D
    srow = alpha * sa * 2.0 ** -14
    return (srow[:, None] * sb[None, :]) * acc
