"""The two-stage eigensolver option (IMCOM_EIGH_TWOSTAGE): dense -> band by
blocked Householder panels, band -> tridiagonal by bulge chasing, then the
same divide and conquer and back-transformations.  It replaces DSYEVR in
imcom_eigen_A (imcom_matrix.f90:617-643) like the one-stage solver, so the
bars are the same: eigenvalues within 1e-12 * lambda_max of LAPACK's,
orthonormal vectors, residual ||AQ - QL|| <= 1e-12 ||A||.  The first stage
alone is checked through imcom_gpu_band_reduce: the band's eigenvalues are
A's (LAPACK dsbevd through scipy as the reference)."""
import numpy as np
import pytest

from imcom_b200 import EIGH_DC, EIGH_TWOSTAGE

from test_gpu_eigen import run_eigen, spectrum_matrix

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _one_stage_after(solver):
    yield
    solver.set_eigensolver(EIGH_DC)


@pytest.mark.parametrize("n", [40, 100, 500])
def test_band_reduction_keeps_the_spectrum(solver, n):
    from scipy.linalg import eig_banded
    A = spectrum_matrix(n, "random", seed=n)
    run_eigen(solver, A, EIGH_DC)  # sets the inputs and loads A
    solver.load_A(A)
    ldb = 33
    AB = np.zeros((n, ldb))
    st = solver.lib.imcom_gpu_band_reduce(solver.h, AB.ctypes.data, ldb)
    assert st == 0
    w_band = eig_banded(np.ascontiguousarray(AB.T), lower=True, eigvals_only=True)
    w = np.linalg.eigvalsh(A)
    assert np.max(np.abs(np.sort(w_band) - w)) < 1e-12 * np.abs(w).max()


@pytest.mark.parametrize("n", [1, 2, 3, 4, 33, 34, 35, 64, 65, 100, 257, 1000])
@pytest.mark.parametrize("kind", ["decay", "cluster", "multiple", "random"])
def test_eigen_twostage(solver, n, kind):
    A = spectrum_matrix(n, kind, seed=n + 1)
    Q, L, _ = run_eigen(solver, A, EIGH_TWOSTAGE)
    ref = np.linalg.eigvalsh(A)[::-1]
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.all(np.diff(L) <= 0)
    assert np.max(np.abs(L - ref)) < 1e-12 * scale
    assert np.max(np.abs(Q.T @ Q - np.eye(n))) < 1e-12
    assert np.max(np.abs(A @ Q - Q * L)) < 1e-12 * scale


def test_twostage_matches_one_stage_on_the_n4096_system(solver):
    """A of the 4 x 32 x 32 headline problem: both solvers' eigenvalues agree
    within 1e-12 lambda_max and the two-stage vectors are orthonormal with
    LAPACK's test ratio <= 10 (checked on the device)."""
    import torch
    from imcom_b200 import synth
    prob = synth.make("n4096", 0)
    solver.set_eigensolver(EIGH_DC)
    solver.set_problem(prob)
    solver.psf_spectra()
    A = solver.build_A()
    _, L1, _ = solver.eigen_A()
    solver.set_eigensolver(EIGH_TWOSTAGE)
    solver.load_A(A)
    Q2, L2, _ = solver.eigen_A()
    assert np.max(np.abs(L1 - L2)) < 1e-12 * L1.max()
    dA, dQ = torch.from_numpy(A).cuda(), torch.from_numpy(Q2).cuda()
    res = torch.linalg.matrix_norm(dA @ dQ - dQ * torch.from_numpy(L2).cuda(), ord=1).item()
    # LAPACK's test ratio ||AQ - Q Lambda||_1 / (n ulp ||A||_1)
    ratio = res / (prob.n * np.finfo(np.float64).eps * torch.linalg.matrix_norm(dA, ord=1).item())
    assert ratio <= 10.0
    orth = (dQ.T @ dQ - torch.eye(prob.n, dtype=torch.float64, device="cuda")).abs().max().item()
    assert orth < 1e-12


def test_twostage_wait_cap_returns_eigen_error(solver):
    """The bulge chase's waits between sweep groups are bounded by the
    eigensolver's iteration cap: a cap of one poll runs out on a system with
    several groups and the call reports the eigensolver error; the same
    context then solves normally."""
    from imcom_b200 import ImcomError
    from imcom_b200.api import OPT_EIGEN_MAXITER
    A = spectrum_matrix(600, "random", seed=3)
    run_eigen(solver, A, EIGH_TWOSTAGE)
    solver.set_option(OPT_EIGEN_MAXITER, 1)
    solver.load_A(A)
    try:
        with pytest.raises(ImcomError) as ei:
            solver.eigen_A()
        assert ei.value.status == 5
        assert "bulge chasing" in str(ei.value)
    finally:
        solver.set_option(OPT_EIGEN_MAXITER, 0)
    solver.load_A(A)
    Q, L, _ = solver.eigen_A()
    assert np.max(np.abs(A @ Q - Q * L)) < 1e-12 * np.abs(L).max()
