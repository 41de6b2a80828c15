"""The learned-kappa features from the neighbour table and the band segments
(IMCOM_OPT_KAPPA_FEATURES = 1, the default; imcom_b200/csrc/kappa.cu) against
the per-pixel scan and element-wise binning (option 0), through the C-ABI: the neighbour
count and exposure count equal, the eight band features equal to float
rounding; and the bracketed bisection's contract -- K and U bit-identical to
the plain bisection -- with the table-built features, also after the inputs
change (the neighbour table is rebuilt).  Each test runs its own context."""
import numpy as np
import pytest

from imcom_b200 import EIGH_DC, EPS, Solver, kappa_model as KM, synth
from imcom_b200.api import OPT_KAPPA_FEATURES

pytestmark = pytest.mark.gpu


def system(s, prob):
    s.set_eigensolver(EIGH_DC)
    s.set_problem(prob)
    C = s.psf_spectra()
    s.build_A(out=False)
    s.eigen_A(out=False)
    s.build_B(out=False)
    s.build_P(out=False)
    return C


@pytest.mark.parametrize("seed", [2, 9])
def test_table_features_equal_scanned_features(seed):
    with Solver(0) as s:
        C = system(s, synth.make("small", seed))
        s.set_option(OPT_KAPPA_FEATURES, 0)
        F0 = s.kappa_features(True, 1e-6, C)
        s.set_option(OPT_KAPPA_FEATURES, 1)
        F1 = s.kappa_features(True, 1e-6, C)
        F2 = s.kappa_features(True, 1e-6, C)  # the cached neighbour table
    assert np.array_equal(F0[:2], F1[:2]) and np.array_equal(F1, F2)
    assert np.max(np.abs(F1[2:10] - F0[2:10]) / np.maximum(1.0, np.abs(F0[2:10]))) < 1e-6
    assert np.array_equal(F0[10:], F1[10:])


def test_learned_bisection_identical_with_table_features():
    model = KM.KappaModel.load(KM.DEFAULT_WEIGHTS)
    us = 1e-6
    with Solver(0) as s:
        s.set_option(OPT_KAPPA_FEATURES, 1)
        for seed in (0, 4):  # a second problem: new inputs, new neighbour table
            C = system(s, synth.make("small", seed))
            kmin, kmax = C * EPS, C / EPS
            tol = us * 1e-3
            K0, U0, _ = s.bisect_kappa(True, us, kmin, kmax, tol, 40, C)
            model.install(s)
            K1, U1, _, _ = s.bisect_kappa_learned(True, us, kmin, kmax, tol, 40, C)
            assert np.array_equal(K0, K1)
            assert np.array_equal(U0, U1)
