"""CPU model of the split-precision product (oracle/split_oracle.py): digit
reconstruction and the error of the product against FP64."""
import numpy as np
import pytest

from oracle import split_oracle as SO


@pytest.mark.parametrize("S", [2, 4, 7, 8])
def test_digits_reconstruct(S):
    rng = np.random.default_rng(S)
    X = rng.standard_normal((40, 300)) * np.exp(rng.uniform(-20, 20, (40, 1)))
    X[3] = 0.0
    d, scale = SO.digits(X, S)
    assert all(np.all(np.abs(p) <= 128) for p in d)
    assert np.all(np.abs(d[0]) <= 65)
    rec = sum(p * 2.0 ** (-7 - 8 * k) for k, p in enumerate(d)) * scale[:, None]
    ulp = 2.0 ** (-7 - 8 * (S - 1))
    # rounding to half a unit of the last digit
    assert np.all(np.abs(rec - X) <= 0.5 * ulp * scale[:, None] * (1 + 1e-12))
    assert scale[3] == 0.0
    live = np.abs(X).max(axis=1) > 0
    r = np.abs(X[live]).max(axis=1) / scale[live]
    assert np.all((r >= 0.25) & (r < 0.5))


@pytest.mark.parametrize("S", [5, 6, 7])
def test_split_product_error_model(S):
    """Error of an element of the split product against an extended-precision
    product: standard deviation below 0.5 sqrt(K) u_S sigma_row sigma_col and
    maximum below 6 sqrt(K) u_S sigma_row sigma_col (the audit assumes a
    standard deviation of 1.0 and bounds of 6 of them)."""
    rng = np.random.default_rng(10 + S)
    K = 1024
    A = rng.standard_normal((96, K))
    B = rng.standard_normal((80, K)) * rng.uniform(0.1, 3, (80, 1))
    C = SO.split_product(A, B, S)
    exact = A.astype(np.longdouble) @ B.T.astype(np.longdouble)
    sa, _ = SO.row_scales(A)
    sb, _ = SO.row_scales(B)
    u = 2.0 ** (-7 - 8 * (S - 1))
    z = ((C - exact) / (np.sqrt(K) * u * sa[:, None] * sb[None, :])).astype(float)
    assert np.sqrt(np.mean(z ** 2)) < 0.5
    assert np.max(np.abs(z)) < 6.0


def test_split_product_exact_for_short_digits():
    """Operands that need only two digits: every dropped diagonal is zero and
    the product is exact up to the final rounding."""
    rng = np.random.default_rng(3)
    A = rng.integers(-2 ** 12, 2 ** 12, (50, 64)).astype(float)
    B = rng.integers(-2 ** 12, 2 ** 12, (30, 64)).astype(float)
    A[:, 0] = 2 ** 13  # fixes every row scale at 2^15: 15 bits per entry
    B[:, 0] = 2 ** 13
    C = SO.split_product(A, B, 4)
    assert np.array_equal(C, A @ B.T)
