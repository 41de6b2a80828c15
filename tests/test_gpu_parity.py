"""GPU solve path (through the C-ABI) against the oracle and the golden
fixtures.  Tolerances: lookup indices are bit-exact by construction (same
floating-point operations), A/B/tables within 1e-12 of the table scale,
eigenvalues within 1e-12 * lambda_max, T and H within 1e-8 relative (normwise),
U and S within 1e-6 relative, kappa within the bisection tolerance."""
import os
import sys

import numpy as np
import pytest

from imcom_b200 import EIGH_DC, EIGH_LIBRARY, EPS, synth
from oracle import oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu

EIG_MODE = int(os.environ.get("IMCOM_TEST_EIGH", EIGH_DC))


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture()
def gs(solver):
    solver.set_eigensolver(EIG_MODE)
    return solver


def oracle_spectra(prob):
    Gt = np.zeros((prob.nps, prob.nps, prob.nexppsf), dtype=np.complex128, order="F")
    for e in range(prob.nexppsf):
        G = prob.G_unrot[:, :, e]
        if abs(prob.rotangdeg[e]) > 2.0 * np.pi * EPS:
            G = O.rotate_image(G, prob.rotangdeg[e])
        Gt[:, :, e] = O.ft_r2c(G)
    return Gt, O.ft_r2c(prob.Gamma)


@pytest.mark.parametrize("case", ["tiny_u", "tiny_rot"])
def test_psf_spectra(gs, case):
    prob, d = make_golden.load(case)
    gs.set_problem(prob)
    C, Gt, Gm = gs.psf_spectra(spectra=True)
    Gt_o, Gm_o = oracle_spectra(prob)
    assert rel(Gt, Gt_o) < 1e-13
    assert rel(Gm, Gm_o) < 1e-13
    assert C == pytest.approx(float(d["C"]), rel=1e-13)
    # exact conjugate fill, as imcom_ft_r2c writes it
    n1 = prob.nps
    assert np.array_equal(Gt[n1 // 2 + 1:, 0, 0], np.conj(Gt[n1 // 2 - 1:0:-1, 0, 0]))


@pytest.mark.parametrize("workload", ["small", "n4096"])
def test_C_is_summed_in_the_reference_order(gs, workload):
    """C_a = sum(|Gammat|^2) / nps^2 rounded as the reference's sequential
    SUM (imcom_matrix.f90:549): the oracle's sequential loop over the GPU's
    own Gammat gives the GPU's C bit for bit (the GPU sums in parallel by
    binades).  At n4096 (nps = 576, 331776 terms) the sequential and the exact
    sums differ by far more than one rounding, so the order is what is
    tested."""
    import math
    prob = synth.make(workload, 0)
    gs.set_problem(prob)
    C, _, Gm = gs.psf_spectra(spectra=True)
    assert C == O.calc_C(Gm)
    t = (Gm.real * Gm.real + Gm.imag * Gm.imag).reshape(-1, order="F")
    exact = math.fsum(t) / prob.nps / prob.nps
    if workload == "n4096":
        assert C != exact


@pytest.mark.parametrize("case", ["tiny_u", "tiny_rot"])
def test_build_A_B(gs, case):
    prob, d = make_golden.load(case)
    gs.set_problem(prob)
    gs.psf_spectra()
    A = gs.build_A()
    B = gs.build_B()
    assert np.array_equal(A, A.T)
    assert rel(A, d["A"]) < 1e-12
    assert rel(B, d["B"]) < 1e-12


def test_build_A_B_small_vs_oracle(gs):
    prob = synth.make("small", 0)
    r = O.solve(prob, UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=40)
    gs.set_problem(prob)
    gs.psf_spectra()
    assert rel(gs.build_A(), r.A) < 1e-12
    assert rel(gs.build_B(), r.B) < 1e-12


def test_eigen_A(gs):
    prob, d = make_golden.load("tiny_u")
    gs.set_inputs(prob.x_i, prob.y_i, prob.exp_i, prob.X_a, prob.Y_a, prob.I_i, None,
                  prob.psfxscale, prob.psfyscale)
    A = d["A"]
    gs.load_A(A)
    Q, L, cond = gs.eigen_A()
    assert np.all(np.diff(L) <= 0)
    assert np.max(np.abs(L - d["L"])) < 1e-12 * d["L"].max()
    assert np.max(np.abs(Q.T @ Q - np.eye(prob.n))) < 1e-12
    assert np.max(np.abs(A @ Q - Q * L)) < 1e-12 * d["L"].max()
    assert cond == pytest.approx(L.max() / L.min())


def _load_system(gs, prob, Q, L, B):
    gs.set_problem(prob)
    gs.load_QL(Q, L)
    gs.load_B(B)


def test_build_P_T_from_oracle_system(gs):
    prob = synth.make("small", 0)
    r = O.solve(prob, UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=40)
    _load_system(gs, prob, r.Q, r.L, r.B)
    P = gs.build_P()
    assert rel(P, r.P) < 1e-13
    gs.load_P(r.P)
    gs.load_K(r.K)
    T = gs.build_T()
    assert rel(T, r.T) < 1e-12


@pytest.mark.parametrize("case", sorted(make_golden.CASES))
def test_bisection_from_oracle_system(gs, case):
    prob, d = make_golden.load(case)
    Q, L, _ = O.eigen_A(d["A"])
    P, P2 = O.build_P(Q, d["B"])
    C = float(d["C"])
    UnotS, US, tol, mx = bool(d["UnotS"]), float(d["US_max"]), float(d["tol"]), int(d["maxnits"])
    Nd = O.build_Ndiag(prob.n, prob.noise)
    K_o, US_o, nev_o = O.bisect_kappa(UnotS, L, P2, Nd, C, US, C * EPS, C / EPS, tol, mx)
    gs.set_problem(prob)
    gs.load_QL(Q, L)
    gs.load_P(P)
    K, USg, nev = gs.bisect_kappa(UnotS, US, C * EPS, C / EPS, tol, mx, C)
    assert np.allclose(K, K_o, rtol=1e-6, atol=0)
    assert np.allclose(USg, US_o, rtol=1e-6)
    assert np.mean(nev == nev_o) > 0.9
    # every accepted kappa meets the target
    ok = nev > 1
    assert np.all(USg[ok] < US)


@pytest.mark.parametrize("case", sorted(make_golden.CASES))
def test_full_solve_vs_golden(gs, case):
    prob, d = make_golden.load(case)
    r = gs.solve(prob, UnotS=bool(d["UnotS"]), US_max=float(d["US_max"]), US_tol=float(d["tol"]),
                 maxnits=int(d["maxnits"]))
    assert np.max(np.abs(r.L - d["L"])) < 1e-12 * d["L"].max()
    assert np.allclose(r.K, d["K"], rtol=1e-6, atol=0)
    assert rel(r.T, d["T"]) < 1e-8
    assert np.allclose(r.U, d["U"], rtol=1e-6)
    assert np.allclose(r.S, d["S"], rtol=1e-6)
    assert rel(r.H, d["H"]) < 1e-8


@pytest.mark.parametrize("UnotS,US,tol", [(True, 1e-6, 1e-8), (False, 0.12, 1e-4)])
def test_full_solve_small_vs_oracle(gs, UnotS, US, tol):
    prob = synth.make("small", 0)
    r_o = O.solve(prob, UnotS=UnotS, US_max=US, US_tol=tol, maxnits=40)
    r = gs.solve(prob, UnotS=UnotS, US_max=US, US_tol=tol, maxnits=40)
    assert np.max(np.abs(r.L - r_o.L)) < 1e-12 * r_o.L.max()
    assert np.allclose(r.K, r_o.K, rtol=1e-6, atol=0)
    assert rel(r.T, r_o.T) < 1e-8
    assert np.allclose(r.U, r_o.U, rtol=1e-6)
    assert np.allclose(r.S, r_o.S, rtol=1e-6)
    assert rel(r.H, r_o.H) < 1e-8


def test_tiny_solve_with_jacobi_vs_oracle(solver):
    """The whole solve of the tiny workload (n = 72) with the one-sided Jacobi
    eigensolver against the oracle (LAPACK DSYEVR inside)."""
    from imcom_b200 import EIGH_DC, EIGH_JACOBI
    from oracle import oracle as Orc
    prob = synth.make("tiny", 4)
    r = Orc.solve(prob, UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=53)
    solver.set_eigensolver(EIGH_JACOBI)
    try:
        g = solver.solve(prob, True, 1e-6, 1e-8, 53)
    finally:
        solver.set_eigensolver(EIGH_DC)
    assert np.max(np.abs(g.K / r.K - 1)) < 1e-6
    assert np.max(np.abs(g.US / r.US - 1)) < 1e-6
    assert np.linalg.norm(g.T - r.T) <= 1e-8 * np.linalg.norm(r.T)
    assert np.linalg.norm(g.H - r.H) <= 1e-8 * np.linalg.norm(r.H)
