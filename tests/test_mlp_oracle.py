"""CPU checks of the MLP oracle used for the GPU gradient check."""
import numpy as np

from oracle import mlp_oracle as M
from imcom_b200 import kappa_model as K


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.14159], dtype=np.float32)
    assert list(M.bf16(x)) == [1.0, 1.0, 1.0 + 2.0 ** -6, -2.5, 3.140625]


def _fd(p, f, t, i, rnd, lt, h=1e-3):
    q1, q2 = p.astype(np.float64), p.astype(np.float64)
    q1[i] += h
    q2[i] -= h
    return (M.loss_and_grad(q1, f, t, rnd, lt)[0] - M.loss_and_grad(q2, f, t, rnd, lt)[0]) / (2 * h)


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = K.init_params(3).astype(np.float64)
    f = rng.standard_normal((12, 64))
    t = rng.standard_normal(64)
    # without rounding the loss is smooth (away from ReLU kinks): every block
    _, g = M.loss_and_grad(p, f, t, round_bf16=False)
    lt = M.loss_and_grad.last_lt  # the width head's target is a constant in the kernel
    for i in [0, 100, 64 * 12 + 5, 64 * 12 + 64 + 77, 64 * 12 + 64 + 4096 + 3, K.NPARAM - 70,
              K.NPARAM - 1]:
        assert abs(_fd(p, f, t, i, False, lt) - g[i]) < 1e-3 * max(1.0, abs(g[i])), i
    # with bf16 rounding the last-layer bias still enters unrounded
    _, gr = M.loss_and_grad(p, f, t)
    ltr = M.loss_and_grad.last_lt
    for i in [K.NPARAM - 1, K.NPARAM - 2]:
        assert abs(_fd(p, f, t, i, True, ltr) - gr[i]) < 1e-3 * max(1.0, abs(gr[i]))


def test_pack_roundtrip():
    p = K.init_params(1)
    assert np.array_equal(K.pack(*K.unpack(p)), p)
    assert p.size == K.NPARAM == 5122
