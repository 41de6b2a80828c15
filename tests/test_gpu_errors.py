"""Error paths of the bounded device waits and iteration caps, made to run out
without faulting or hanging the GPU.

Each test makes one bounded wait or cap run out on purpose -- a grid barrier
that waits for an arrival nothing makes, a split-GEMM pipeline whose copy
producer issues nothing, a secular-equation solver capped at one iteration --
checks that the call returns the documented status (the reference stops with
a message where LAPACK reports info > 0, imcom_matrix.f90:645-653), then
clears the option and checks that the same context solves normally again.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

IMCOM_ERR_EIGEN, IMCOM_ERR_SPLIT = 5, 9
KW = dict(UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=40)


@pytest.fixture(scope="module")
def prob():
    from imcom_b200 import synth
    return synth.make("small", seed=0)


def _fresh():
    from imcom_b200 import EIGH_DC, Solver
    s = Solver(0)
    s.set_eigensolver(EIGH_DC)
    return s


def _eig_check(prob_A, Q, L):
    A = prob_A
    scale = np.linalg.norm(A, 2)
    assert np.linalg.norm(A @ Q - Q * L, 2) <= 1e-11 * scale
    assert np.abs(Q.T @ Q - np.eye(len(L))).max() <= 1e-11


def test_tridiagonalisation_barrier_timeout_returns_eigen_error(prob):
    from imcom_b200 import ImcomError
    from imcom_b200.api import OPT_EIGEN_MAXITER, OPT_STALL_TEST, OPT_TAIL_CTAS, STALL_TRIDIAG

    with _fresh() as s:
        s.set_option(OPT_TAIL_CTAS, -1)  # panels all the way: the grid barrier runs
        s.set_problem(prob)
        s.psf_spectra()
        A = s.build_A()
        s.set_option(OPT_EIGEN_MAXITER, 20000)
        s.set_option(OPT_STALL_TEST, STALL_TRIDIAG)
        with pytest.raises(ImcomError) as ei:
            s.eigen_A()
        assert ei.value.status == IMCOM_ERR_EIGEN
        assert "barrier" in str(ei.value)
        # the same context, the option cleared: a normal decomposition
        s.set_option(OPT_STALL_TEST, 0)
        s.set_option(OPT_EIGEN_MAXITER, 0)
        s.load_A(A)
        Q, L, _ = s.eigen_A()
        _eig_check(A, Q, L)


def test_divide_and_conquer_iteration_cap_returns_eigen_error(prob):
    from imcom_b200 import ImcomError
    from imcom_b200.api import OPT_DC_MAXITER

    with _fresh() as s:
        s.set_problem(prob)
        s.psf_spectra()
        A = s.build_A()
        s.set_option(OPT_DC_MAXITER, 1)
        with pytest.raises(ImcomError) as ei:
            s.eigen_A()
        assert ei.value.status == IMCOM_ERR_EIGEN
        assert "divide and conquer" in str(ei.value)
        s.set_option(OPT_DC_MAXITER, 0)
        s.load_A(A)
        Q, L, _ = s.eigen_A()
        _eig_check(A, Q, L)


def test_split_pipeline_wait_timeout_returns_split_error(prob):
    from imcom_b200 import ImcomError
    from imcom_b200.api import OPT_STALL_TEST, STALL_SPLIT

    with _fresh() as s:
        s.set_precision(True)
        ref = s.solve(prob, **KW)
        s.set_option(OPT_STALL_TEST, STALL_SPLIT)
        kmin, kmax = ref.kappa_min, ref.kappa_max
        s.build_P(out=False)  # queued; the wait runs out on the device (2 s)
        with pytest.raises(ImcomError) as ei:
            s.bisect_kappa(True, KW["US_max"], kmin, kmax, KW["US_tol"], KW["maxnits"])
        assert ei.value.status == IMCOM_ERR_SPLIT
        assert "wait ran out" in str(ei.value)
        s.set_option(OPT_STALL_TEST, 0)
        again = s.solve(prob, **KW)
        assert np.array_equal(again.K, ref.K)
        assert np.max(np.abs(again.T - ref.T)) <= 1e-12 * np.abs(ref.T).max()


def test_stall_option_rejects_unknown_bits():
    from imcom_b200 import ImcomError
    from imcom_b200.api import OPT_STALL_TEST

    with _fresh() as s:
        with pytest.raises(ImcomError) as ei:
            s.set_option(OPT_STALL_TEST, 4)
        assert ei.value.status == -3
