"""GPU solve path against the oracle at the headline sizes and on the
reference's own example case.

* n4096 (4 x 32 x 32 inputs, Airy PSFs, 64 x 64 outputs; seed 0): the whole
  solve through the C-ABI, plain FP64 and learned kappa + split-precision P/T,
  at U < 1e-2 (tolerance 1e-5, the benchmark's target) and at U < 1e-6
  (tolerance 1e-8), against one oracle solve (LAPACK DSYEVR inside).  Bars:
  eigenvalues within 1e-12 lambda_max, kappa within 1e-6 relative (the
  bisection's own resolution is coarser), U and S within 1e-6 relative, T
  within 1e-8 relative (largest element and every column), H within 1e-8
  (normwise).  The eigendecomposition alone is also checked against LAPACK's
  at this size (eigenvalues, orthogonality, and the residual as LAPACK's own
  test ratio ||AQ - Q Lambda||_1 / (n ulp ||A||_1) <= 10).
* n16200 (8 x 45 x 45 inputs, 128 x 128 outputs): stage by stage on the GPU's
  own results -- A Q = Q Lambda and Q^T Q = I (formed on the device with
  torch as the checker), P = Q^T B and T columns on 64 seeded pixels against
  numpy / the oracle's build_T, and the oracle's bisection on every pixel
  from the GPU's L and P against the GPU's kappa and U.
* Three patches of the batched workload (the largest n = 2269, the median and
  the smallest n = 990 of the benchmark's 256) against the oracle.
* The reference's documented example (example/userxy1/config_example run as
  ``./imcom config_example S 1.d-3 1.d-6``): read through this library's
  configuration and FITS readers, solved on the GPU (plain and split) and by
  the oracle, compared at the bars above; H is also compared with the truth
  image the reference ships (ideal_output.example.fits), the reference's own
  qualitative check.
"""
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_example_fixture  # noqa: E402

pytestmark = pytest.mark.gpu

TOLS = {"U1e-2": (True, 1e-2, 1e-5), "U1e-6": (True, 1e-6, 1e-8)}


def relmax(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def scaled(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def column_rel(a, b):
    nb = np.linalg.norm(b, axis=0)
    return float(np.max(np.linalg.norm(a - b, axis=0) / np.maximum(nb, 1e-300)))


def oracle_at(r, prob, UnotS, US, tol, maxnits=53):
    """The oracle's bisection, T and maps on an oracle system `r`."""
    K, USo, nev = O.bisect_kappa(UnotS, r.L, r.P2, r.Ndiag, r.C_a, US, r.kappa_min, r.kappa_max,
                                 tol, maxnits)
    T = O.build_T(r.Q, r.P, r.L, K)
    out = {"K": K, "US": USo, "nev": nev, "T": T, "H": O.build_image(T, prob.I_i)}
    if UnotS:
        out["U"], out["S"] = USo, O.build_S(T, r.Ndiag)
    else:
        out["S"], out["U"] = USo, O.build_U(r.L, r.P2, r.C_a, K)
    return out


# LAPACK's own test of an eigendecomposition (dsyt21): ||A Q - Q Lambda||_1 /
# (n ulp ||A||_1); LAPACK's test drivers accept ratios below their threshold
# (tens).  The bar here is 10.
RATIO_BAR = 10.0


def residual_ratio(res_1norm, a_1norm, n):
    return res_1norm / (n * np.finfo(np.float64).eps * a_1norm)


def check_solve(g, o, L_o):
    assert np.max(np.abs(g.L - L_o)) <= 1e-12 * L_o.max()
    assert relmax(g.K, o["K"]) <= 1e-6
    assert relmax(g.U, o["U"]) <= 1e-6
    assert relmax(g.S, o["S"]) <= 1e-6
    assert scaled(g.T, o["T"]) <= 1e-8
    assert column_rel(g.T, o["T"]) <= 1e-8
    assert np.linalg.norm(g.H - o["H"]) <= 1e-8 * np.linalg.norm(o["H"])


def set_fast(solver, fast):
    from imcom_b200 import EIGH_DC
    solver.set_eigensolver(EIGH_DC)
    solver.set_precision(bool(fast))
    if fast:
        from imcom_b200 import kappa_model as KM
        KM.KappaModel.load(KM.DEFAULT_WEIGHTS).install(solver)


# ---- n4096 ----------------------------------------------------------------

@pytest.fixture(scope="module")
def n4096():
    from imcom_b200 import synth
    prob = synth.make("n4096", 0)
    r = O.solve(prob, UnotS=True, US_max=1e-2, US_tol=1e-5, maxnits=53, keep_tables=False)
    return prob, r, {k: oracle_at(r, prob, *v) for k, v in TOLS.items()}


@pytest.mark.parametrize("tol", sorted(TOLS))
@pytest.mark.parametrize("fast", [False, True], ids=["plain_fp64", "learned_split"])
def test_n4096_full_solve_vs_oracle(solver, n4096, fast, tol):
    prob, r, ref = n4096
    UnotS, US, t = TOLS[tol]
    set_fast(solver, fast)
    try:
        g = solver.solve(prob, UnotS=UnotS, US_max=US, US_tol=t, maxnits=53, learned=fast,
                         keep=("Q", "T"))
    finally:
        solver.set_precision(False)
    check_solve(g, ref[tol], r.L)
    # the bisection takes the oracle's decisions: evaluation counts agree
    assert np.mean(g.nevals == ref[tol]["nev"]) >= 0.99 or fast


def test_n4096_eigen_vs_lapack(solver, n4096):
    prob, r, _ = n4096
    from imcom_b200 import EIGH_DC
    solver.set_eigensolver(EIGH_DC)
    solver.set_problem(prob)
    solver.load_A(r.A)
    Q, L, cond = solver.eigen_A()
    lmax = r.L.max()
    assert np.max(np.abs(L - r.L)) <= 1e-12 * lmax
    assert cond == pytest.approx(L.max() / L.min())
    import torch
    dQ = torch.from_numpy(Q).cuda()
    dA = torch.from_numpy(r.A).cuda()
    res = torch.linalg.matrix_norm(dA @ dQ - dQ * torch.from_numpy(L).cuda(), ord=1).item()
    orth = (dQ.T @ dQ - torch.eye(prob.n, dtype=torch.float64, device="cuda")).abs().max().item()
    assert residual_ratio(res, torch.linalg.matrix_norm(dA, ord=1).item(), prob.n) <= RATIO_BAR
    assert orth <= 1e-12
    # the eigenvectors of well-separated eigenvalues agree with LAPACK's up to sign
    gap = np.minimum(np.abs(np.diff(r.L, prepend=np.inf)), np.abs(np.diff(r.L, append=-np.inf)))
    sep = np.nonzero(gap > 1e-6 * lmax)[0][:64]
    dots = np.abs(np.sum(Q[:, sep] * r.Q[:, sep], axis=0))
    assert np.all(dots >= 1 - 1e-9)


# ---- n16200, stage by stage ---------------------------------------------------

def test_n16200_stages_vs_oracle(solver):
    import torch

    from imcom_b200 import EIGH_DC, synth
    from imcom_b200.problem import build_Ndiag
    prob = synth.make("n16200", 0)
    UnotS, US, tol = True, 1e-6, 1e-8
    solver.set_eigensolver(EIGH_DC)
    solver.set_precision(False)
    g = solver.solve(prob, UnotS=UnotS, US_max=US, US_tol=tol, maxnits=53,
                     keep=("A", "B", "Q", "P", "T"))
    n, m = prob.n, prob.m
    # eigendecomposition residual and orthogonality (checker on the device)
    dQ = torch.from_numpy(g.Q).cuda()
    dA = torch.from_numpy(g.A).cuda()
    dL = torch.from_numpy(g.L).cuda()
    res = torch.linalg.matrix_norm(dA @ dQ - dQ * dL, ord=1).item()
    assert residual_ratio(res, torch.linalg.matrix_norm(dA, ord=1).item(), n) <= RATIO_BAR
    orth = (dQ.T @ dQ - torch.eye(n, dtype=torch.float64, device="cuda")).abs().max().item()
    assert orth <= 1e-12
    assert np.all(np.diff(g.L) <= 0)
    del dA, dQ, dL
    torch.cuda.empty_cache()
    # P and T columns on a seeded sample of pixels
    cols = np.sort(np.random.default_rng(7).choice(m, 64, replace=False))
    P_s = g.Q.T @ g.B[:, cols]
    assert scaled(g.P[:, cols], P_s) <= 1e-12
    T_s = O.build_T(g.Q, g.P[:, cols], g.L, g.K[cols])
    assert column_rel(g.T[:, cols], T_s) <= 1e-10
    # the oracle's bisection on the GPU's L and P, every pixel
    Nd = build_Ndiag(n, prob.noise)
    K_o, US_o, nev_o = O.bisect_kappa(UnotS, g.L, g.P * g.P, Nd, g.C_a, US, g.kappa_min,
                                      g.kappa_max, tol, 53)
    assert relmax(g.K, K_o) <= 1e-6
    assert relmax(g.US, US_o) <= 1e-6
    assert np.mean(g.nevals == nev_o) >= 0.99


# ---- batched-workload patches -------------------------------------------------

def bench_patch(i, npatch=256, seed0=1000):
    """Patch i of the benchmark's batched workload (imcom_b200.batch.make_batch)."""
    from imcom_b200 import synth
    sides = np.random.default_rng(seed0).integers(16, 25, npatch)
    return synth.make_patch(seed=seed0 + i, side=int(sides[i]))


@pytest.mark.parametrize("i,n", [(91, 2269), (8, 1562), (224, 990)],
                         ids=["largest", "median", "smallest"])
def test_batch_patches_vs_oracle(solver, i, n):
    from imcom_b200 import EIGH_DC
    p = bench_patch(i)
    assert p.n == n
    KW = dict(UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=53)
    r = O.solve(p, keep_tables=False, **KW)
    solver.set_eigensolver(EIGH_DC)
    solver.set_precision(False)
    g = solver.solve(p, keep=("T",), **KW)
    ref = {"K": r.K, "U": r.U, "S": r.S, "T": r.T, "H": r.H}
    check_solve(g, ref, r.L)


# ---- the reference's example case ---------------------------------------------

# The documented run (Sigma < 1e-3, tolerance 1e-6) and a strict leakage
# target (U < 1e-6, tolerance 1e-8) at which H reproduces the truth image.
EXAMPLE_RUNS = {"S1e-3": (False, 1e-3, 1e-6), "U1e-6": (True, 1e-6, 1e-8)}
# rms of H - ideal over the central 49 x 49 output pixels, relative to the
# ideal image's rms, at U < 1e-6: the oracle's own solve gives 1.4e-5
EXAMPLE_RMS = 5e-5


def lapack_spread(r, prob, ref):
    """How far the reference's own results move with the eigensolver: the
    same solve on dsyevd's eigenpairs (numpy) instead of dsyevr's, of A and of
    A plus a seeded symmetric perturbation with ||dA||_1 = n eps ||A||_1 (the
    backward error of a solver at LAPACK's test ratio 1), per run, as the
    larger (S relmax, T column relmax) over the pixels at kappa_min.  There U
    and T are set by eigenmodes whose eigenvalues are at the rounding level of
    A, which no two eigensolvers share; the GPU solver's own result there
    varies between runs (its reductions add partial sums in arrival order).
    Returns (S relmax, T column relmax, U relmax) per run."""
    from types import SimpleNamespace
    n = r.A.shape[0]
    rng = np.random.default_rng(11)
    E = rng.standard_normal((n, n))
    E = E + E.T
    norm1 = lambda M: np.abs(M).sum(axis=0).max()
    E *= n * np.finfo(np.float64).eps * norm1(r.A) / norm1(E)
    out = {k: (0.0, 0.0, 0.0) for k in EXAMPLE_RUNS}
    for A in (r.A, r.A + E):
        w, V = np.linalg.eigh(A)
        L2, Q2 = w[::-1].copy(), V[:, ::-1].copy()
        P2 = Q2.T @ r.B
        alt = SimpleNamespace(L=L2, Q=Q2, P=P2, P2=P2 * P2, Ndiag=r.Ndiag, C_a=r.C_a,
                              kappa_min=r.kappa_min, kappa_max=r.kappa_max)
        for k, v in EXAMPLE_RUNS.items():
            a, o = oracle_at(alt, prob, *v), ref[k]
            at_min = o["K"] <= r.kappa_min
            if at_min.any():
                out[k] = (max(out[k][0], relmax(a["S"][at_min], o["S"][at_min])),
                          max(out[k][1], column_rel(a["T"][:, at_min], o["T"][:, at_min])),
                          max(out[k][2], relmax(a["U"][at_min], o["U"][at_min])))
    return out


@pytest.fixture(scope="module")
def example(tmp_path_factory):
    from imcom_b200 import config, fits
    d = str(tmp_path_factory.mktemp("userxy1"))
    path = make_example_fixture.unpack(d)
    prob = config.load_problem(path)
    r = O.solve(prob, UnotS=False, US_max=1e-3, US_tol=1e-6, maxnits=53, keep_tables=False)
    ref = {k: oracle_at(r, prob, *v) for k, v in EXAMPLE_RUNS.items()}
    ideal = fits.read(os.path.join(d, "ideal_output.example.fits")).reshape(-1, order="F")
    return prob, r, ref, ideal, lapack_spread(r, prob, ref)


def test_example_config_reads_like_the_reference(example):
    prob, r, ref, ideal, _ = example
    assert (prob.n, prob.m, prob.n1out, prob.n2out) == (4096, 4225, 65, 65)
    # equal rotations: imcom_test_psfconst reports "not constant" (its quirk)
    assert prob.psfconst == 0 and prob.nexppsf == 4
    assert prob.nps == 640  # 2 nint(32 / 0.1), above twice the 256-pixel PSF stamp
    assert ideal.shape == (4225,)


def central_rms(H, ideal):
    Hc = H.reshape(65, 65, order="F")[8:-8, 8:-8]
    Ic = ideal.reshape(65, 65, order="F")[8:-8, 8:-8]
    return float(np.sqrt(np.mean((Hc - Ic) ** 2)) / np.sqrt(np.mean(Ic ** 2)))


@pytest.mark.parametrize("run", sorted(EXAMPLE_RUNS))
@pytest.mark.parametrize("fast", [False, True], ids=["plain_fp64", "split"])
def test_example_solve_vs_oracle(solver, example, fast, run):
    """The bars on every pixel with kappa > kappa_min; at kappa_min (129
    pixels of the U < 1e-6 run) S, T and U within the spread of the
    reference's own results between two LAPACK drivers and under a backward
    error of n eps ||A||_1 (S 1.8e-3, T 1.0e-2, U 1.5e-6 when measured; the
    two drivers alone, which share one Householder reduction, differ by 4e-5
    to 1.1e-4 in S and 5e-4 in T), where the reference itself is not
    reproducible to the bars."""
    prob, r, ref, ideal, spread = example
    UnotS, US, tol = EXAMPLE_RUNS[run]
    from imcom_b200 import EIGH_DC
    solver.set_eigensolver(EIGH_DC)
    solver.set_precision(fast)
    try:
        g = solver.solve(prob, UnotS=UnotS, US_max=US, US_tol=tol, maxnits=53, keep=("T",))
    finally:
        solver.set_precision(False)
    from types import SimpleNamespace
    o = ref[run]
    at_min = o["K"] <= r.kappa_min
    keep = ~at_min
    check_solve(SimpleNamespace(L=g.L, H=g.H, K=g.K[keep], U=g.U[keep], S=g.S[keep],
                                T=g.T[:, keep]),
                dict(K=o["K"][keep], U=o["U"][keep], S=o["S"][keep], T=o["T"][:, keep],
                     H=o["H"]), r.L)
    assert relmax(g.K, o["K"]) <= 1e-6 and relmax(g.U[keep], o["U"][keep]) <= 1e-6
    if at_min.any():
        s_spread, t_spread, u_spread = spread[run]
        assert relmax(g.U[at_min], o["U"][at_min]) <= max(1e-6, u_spread)
        assert relmax(g.S[at_min], o["S"][at_min]) <= max(1e-6, s_spread)
        assert column_rel(g.T[:, at_min], o["T"][:, at_min]) <= max(1e-8, t_spread)
    # every accepted kappa keeps U (or Sigma) below the target
    assert np.all(g.US[g.nevals > 1] < US)
    if UnotS:
        # the reference's qualitative check: H reproduces the ideal output
        # image away from the borders
        assert central_rms(g.H, ideal) <= EXAMPLE_RMS
        assert central_rms(ref[run]["H"], ideal) <= EXAMPLE_RMS
