"""The own FP64 eigensolver (tridiagonalisation + divide and conquer +
back-transformation) on matrices with IMCOM-like spectra: decades of decay,
near-degenerate clusters, exact multiplicities and tiny sizes.  Reference:
LAPACK through numpy; parity bars as for imcom_eigen_A: eigenvalues within
1e-12 * lambda_max, orthonormal vectors, residual ||AQ - QL|| <= 1e-12 ||A||."""
import numpy as np
import pytest

from imcom_b200 import EIGH_DC, EIGH_LIBRARY

pytestmark = pytest.mark.gpu


def spectrum_matrix(n, kind, seed):
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    if kind == "decay":
        lam = np.logspace(-1, -16, n)
    elif kind == "cluster":
        lam = np.concatenate([np.logspace(-1, -13, n - n // 2),
                              1e-3 * (1 + 1e-13 * rng.standard_normal(n // 2))])
    elif kind == "multiple":
        lam = np.repeat(rng.random(max(1, n // 8)), 8)[:n]
        lam = np.concatenate([lam, np.ones(n - len(lam))])
    else:
        lam = rng.standard_normal(n)
    A = (Q * lam) @ Q.T
    return np.asfortranarray(0.5 * (A + A.T))


def run_eigen(solver, A, mode):
    n = A.shape[0]
    x = np.arange(n, dtype=float)
    solver.set_inputs(x, x, np.ones(n, dtype=np.int32), x[:1], x[:1], None, None, 1.0, 1.0)
    solver.set_eigensolver(mode)
    solver.load_A(A)
    return solver.eigen_A()


@pytest.mark.parametrize("n", [1, 2, 3, 31, 33, 72, 257, 1000])
@pytest.mark.parametrize("kind", ["decay", "cluster", "multiple", "random"])
def test_eigen_dc(solver, n, kind):
    A = spectrum_matrix(n, kind, seed=n)
    Q, L, cond = run_eigen(solver, A, EIGH_DC)
    ref = np.linalg.eigvalsh(A)[::-1]
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.all(np.diff(L) <= 0)
    assert np.max(np.abs(L - ref)) < 1e-12 * scale
    assert np.max(np.abs(Q.T @ Q - np.eye(n))) < 1e-12
    assert np.max(np.abs(A @ Q - Q * L)) < 1e-12 * scale


def test_eigen_dc_matches_library_n2048(solver):
    A = spectrum_matrix(2048, "cluster", seed=7)
    Q1, L1, _ = run_eigen(solver, A, EIGH_DC)
    Q2, L2, _ = run_eigen(solver, A, EIGH_LIBRARY)
    assert np.max(np.abs(L1 - L2)) < 1e-12 * L2.max()
    assert np.max(np.abs(A @ Q1 - Q1 * L1)) < 1e-12 * L2.max()
    assert np.max(np.abs(Q1.T @ Q1 - np.eye(2048))) < 1e-12


@pytest.mark.parametrize("tail", [0, -1])
def test_tridiagonalisation_graph_replay(solver, tail):
    """The first eigensolve at a size runs the tridiagonalisation's launches
    directly, the second captures them into a CUDA graph and the third
    replays it (with and without the cluster tail): all three meet the parity
    bars, and each adds the same number of launches to the library's
    counter."""
    from imcom_b200.api import OPT_TAIL_CTAS
    A = spectrum_matrix(1500, "decay", seed=3)
    solver.set_option(OPT_TAIL_CTAS, tail)
    try:
        out, counts = [], []
        for _ in range(3):
            c0 = solver.launch_count()
            out.append(run_eigen(solver, A, EIGH_DC))
            counts.append(solver.launch_count() - c0)
    finally:
        solver.set_option(OPT_TAIL_CTAS, 0)
    ref = np.linalg.eigvalsh(A)[::-1]
    scale = np.abs(ref).max()
    for Q, L, _ in out:
        assert np.max(np.abs(L - ref)) < 1e-12 * scale
        assert np.max(np.abs(A @ Q - Q * L)) < 1e-12 * scale
        assert np.max(np.abs(Q.T @ Q - np.eye(A.shape[0]))) < 1e-12
    assert counts[0] == counts[1] == counts[2]


@pytest.mark.parametrize("n", [1, 2, 3, 31, 33, 72, 112])
@pytest.mark.parametrize("kind", ["decay", "cluster", "multiple"])
def test_eigen_jacobi(solver, n, kind):
    """The one-sided Jacobi eigensolver (IMCOM_EIGH_JACOBI, n <= 112) on the
    positive semi-definite spectra, to the same bars as the D&C solver."""
    from imcom_b200 import EIGH_JACOBI
    A = spectrum_matrix(n, kind, seed=n)
    try:
        Q, L, _ = run_eigen(solver, A, EIGH_JACOBI)
    finally:
        solver.set_eigensolver(EIGH_DC)
    ref = np.linalg.eigvalsh(A)[::-1]
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.all(np.diff(L) <= 0)
    assert np.max(np.abs(L - ref)) < 1e-12 * scale
    assert np.max(np.abs(Q.T @ Q - np.eye(n))) < 1e-12
    assert np.max(np.abs(A @ Q - Q * L)) < 1e-12 * scale


def test_eigh_jacobi_batched(solver):
    """Many small systems in one launch (one thread block each): every
    matrix of the stack meets the bars; n above the limit is rejected."""
    from imcom_b200 import ImcomError
    mats = [spectrum_matrix(64, kind, seed=s) for s in range(4)
            for kind in ("decay", "cluster", "multiple")]
    Q, L, sweeps = solver.eigh_jacobi_batched(np.stack(mats))
    assert Q.shape == (12, 64, 64) and L.shape == (12, 64)
    assert np.all(sweeps > 0)
    for A, Qb, Lb in zip(mats, Q, L):
        ref = np.linalg.eigvalsh(A)
        scale = np.abs(ref).max()
        assert np.all(np.diff(Lb) >= 0)
        assert np.max(np.abs(Lb - ref)) < 1e-12 * scale
        assert np.max(np.abs(Qb.T @ Qb - np.eye(64))) < 1e-12
        assert np.max(np.abs(A @ Qb - Qb * Lb)) < 1e-12 * scale
    with pytest.raises(ImcomError):
        solver.eigh_jacobi_batched(np.eye(113))
