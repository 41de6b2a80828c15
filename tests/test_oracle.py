"""The CPU oracle against known answers and against the independent numpy
mirror's golden fixtures (tests/golden).  No GPU needed."""
import math
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O
from imcom_b200 import synth

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402

EPS = 1.1102230246251565e-16


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


# ---- DLAMCH ---------------------------------------------------------------
def test_dlamch():
    assert O.dlamch("E") == EPS
    assert O.dlamch("S") == np.finfo(np.float64).tiny


# ---- FFT (stand-in for FFTW) ---------------------------------------------
@pytest.mark.parametrize("shape", [(8, 8), (12, 10), (22, 33), (96, 96), (15, 7)])
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft2d_matches_numpy(shape, sign):
    rng = np.random.default_rng(shape[0] * 100 + shape[1])
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    ref = np.fft.fft2(a) if sign < 0 else np.fft.ifft2(a) * a.size
    assert rel(O.fft2d(a, sign), ref) < 1e-14


@pytest.mark.parametrize("shape", [(16, 16), (20, 14), (21, 15)])
def test_ft_r2c_full_hermitian(shape):
    r = np.random.default_rng(1).standard_normal(shape)
    F = O.ft_r2c(r)
    assert rel(F, np.fft.fft2(r)) < 1e-14
    n1, n2 = shape
    # the filled half is the exact conjugate mirror (imcom_proc.f90:459-473)
    for k in range(n1 // 2 + 1, n1):
        for j in range(n2):
            assert F[k, j] == np.conj(F[n1 - k, (n2 - j) % n2])


# ---- Neville (imcom_polint / imcom_polin2) -------------------------------
def test_polint_reproduces_degree7():
    rng = np.random.default_rng(3)
    c = rng.standard_normal(8)
    xa = np.arange(11.0, 19.0)
    for x in (11.0, 13.25, 14.5, 17.9, 18.0):
        assert O.polint(xa, np.polyval(c, xa), x) == pytest.approx(np.polyval(c, x), rel=1e-12)


def test_polint_trap_on_duplicate_abscissae():
    with pytest.raises(ValueError):
        O.polint([1.0, 1.0, 2.0], [0.0, 1.0, 2.0], 1.5)


def test_interp_lookup_window_indices():
    L = 40
    tab = np.random.default_rng(0).standard_normal((L, L))
    rng = np.random.default_rng(1)
    for _ in range(200):
        xarg, yarg = rng.uniform(-25, 25, 2)
        if rng.random() < 0.2:
            xarg = float(round(xarg))
        v, win, st = O.interp_lookup(tab, xarg, yarg)
        iarg, jarg = L // 2 + 1 + xarg, L // 2 + 1 + yarg
        fi, ci, fj, cj = math.floor(iarg), math.ceil(iarg), math.floor(jarg), math.ceil(jarg)
        inside = fi >= 1 and fj >= 1 and ci <= L and cj <= L
        if not inside:
            assert v == 0.0 and list(win) == [0, 0, 0, 0]
            continue
        assert list(win) == [max(1, fi - 3), min(L, ci + 3), max(1, fj - 3), min(L, cj + 3)]


# ---- tables: exact identities of the zero-padded DFT -----------------------
def test_Alookup_integer_shifts_are_circular_autocorrelation():
    prob = synth.make("tiny", 0)
    G = prob.G_unrot[:, :, 0]
    Gt = np.asfortranarray(np.stack([O.ft_r2c(G)], axis=2))
    tab = O.build_Alookup(Gt, npad=3)[:, :, 0]
    nps = G.shape[0]
    L = 3 * nps
    c = L // 2  # 0-based centre (L/2 + 1, 1-based)
    scale = np.abs(tab).max()
    for s in [(0, 0), (1, 0), (0, 2), (3, -1), (-4, 5)]:
        ref = np.sum(G * np.roll(G, (-s[0], -s[1]), axis=(0, 1)))
        assert abs(tab[c + 3 * s[0], c + 3 * s[1]] - ref) < 1e-13 * scale


def test_Blookup_is_minus_two_cross_correlation():
    prob = synth.make("tiny", 0)
    G = prob.G_unrot[:, :, 0]
    Gt = np.asfortranarray(O.ft_r2c(G)[:, :, None])
    Gm = O.ft_r2c(prob.Gamma)
    tab = O.build_Blookup(Gt, Gm, npad=3)[:, :, 0]
    L = 3 * G.shape[0]
    c = L // 2
    scale = np.abs(tab).max()
    for s in [(0, 0), (2, 1), (-3, 0)]:
        ref = -2.0 * np.sum(prob.Gamma * np.roll(G, (-s[0], -s[1]), axis=(0, 1)))
        assert abs(tab[c + 3 * s[0], c + 3 * s[1]] - ref) < 1e-13 * scale


def test_calc_C_is_parseval():
    prob = synth.make("tiny", 0)
    assert O.calc_C(O.ft_r2c(prob.Gamma)) == pytest.approx(np.sum(prob.Gamma ** 2), rel=1e-13)


def test_rotate_image_conserves_flux_and_symmetry():
    # Gaussian centred on the rotation centre ((n+1)/2, 1-based)
    x = np.arange(1, 49) - 24.5
    g = np.asfortranarray(np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / (2 * 6.4 ** 2)))
    r = O.rotate_image(g, 30.0)
    assert r.sum() == pytest.approx(g.sum(), rel=1e-13)
    inner = slice(8, 40)
    # edge pixels whose source leaves the image become 0 and the flux rescale
    # (imcom_proc.f90:249) lifts the rest by ~1e-4 for this Gaussian
    assert np.abs(r[inner, inner] - g[inner, inner]).max() < 1e-3 * g.max()


# ---- Ndiag quirk, eigen, P, T ----------------------------------------------
def test_build_Ndiag_contiguous_blocks():
    nd = O.build_Ndiag(10, [1.0, 2.0, 3.0])
    assert list(nd) == [1, 1, 1, 2, 2, 2, 3, 3, 3, 3]


def test_eigen_A_descending_and_T_identity():
    prob, d = make_golden.load("tiny_u")
    A = d["A"]
    Q, L, cond = O.eigen_A(A)
    assert np.all(np.diff(L) <= 0)
    assert rel(L, np.linalg.eigvalsh(A)[::-1]) < 1e-12
    assert cond == pytest.approx(L.max() / L.min())
    B = d["B"]
    P, P2 = O.build_P(Q, B)
    K = np.full(prob.m, 1e-6)
    T = O.build_T(Q, P, L, K)
    ref = -0.5 * np.linalg.solve(A + 1e-6 * np.eye(prob.n), B)
    assert rel(T, ref) < 1e-8


# ---- full solve against the independent mirror (golden fixtures) -----------
@pytest.mark.parametrize("case", sorted(make_golden.CASES))
def test_oracle_matches_numpy_mirror(case):
    prob, d = make_golden.load(case)
    r = O.solve(prob, UnotS=bool(d["UnotS"]), US_max=float(d["US_max"]), US_tol=float(d["tol"]),
                maxnits=int(d["maxnits"]))
    assert r.C_a == pytest.approx(float(d["C"]), rel=1e-13)
    assert rel(r.A, d["A"]) < 1e-13
    assert rel(r.B, d["B"]) < 1e-13
    assert np.max(np.abs(r.L - d["L"])) < 1e-12 * d["L"].max()
    assert np.allclose(r.K, d["K"], rtol=1e-6, atol=0)
    assert rel(r.T, d["T"]) < 1e-8
    assert np.allclose(r.U, d["U"], rtol=1e-6)
    assert np.allclose(r.S, d["S"], rtol=1e-6)
    assert rel(r.H, d["H"]) < 1e-8


def test_bisection_contract():
    prob, d = make_golden.load("tiny_u")
    L, P = d["L"], None
    Q, Lo, _ = O.eigen_A(d["A"])
    P, P2 = O.build_P(Q, d["B"])
    C = float(d["C"])
    kmin, kmax = C * EPS, C / EPS
    K, U, nev = O.bisect_kappa(True, Lo, P2, O.build_Ndiag(prob.n, prob.noise), C, 1e-4, kmin,
                               kmax, 1e-7, 40)
    for a in range(prob.m):
        u0 = O.U_from_kappa(Lo, P2[:, a], C, kmin)
        if u0 >= 1e-4:
            assert K[a] == kmin and nev[a] == 1
        else:
            assert U[a] < 1e-4
            assert O.U_from_kappa(Lo, P2[:, a], C, K[a]) == pytest.approx(U[a], rel=1e-9)
            assert nev[a] <= 41
