"""ctypes wrapper of the CPU oracle (test infrastructure only).

Each function mirrors one reference subroutine (file:line in the docstring of
``imcom_oracle.cpp``).  Arrays are numpy, Fortran (column-major) order,
float64 / int32.  ``solve`` replays the build branch of the reference driver
(imcom.f90:90-169) on in-memory inputs.

Only tests/, ``__graft_entry__.smoke`` and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

_lib = None

_d = C.c_double
_i = C.c_int
_p = C.c_void_p


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(path)
        sig = {
            "oracle_set_threads": (None, [_i]),
            "oracle_get_threads": (_i, []),
            "oracle_dlamch": (_d, [C.c_char_p]),
            "oracle_fft2d": (None, [_i, _i, _i, _p]),
            "oracle_polint": (_i, [_i, _p, _p, _d, _p]),
            "oracle_rotate_image": (_i, [_i, _i, _p, _d, _i, _i, _p]),
            "oracle_ft_r2c": (None, [_i, _i, _p, _p]),
            "oracle_build_Alookup": (None, [_i, _i, _i, _p, _p]),
            "oracle_build_Blookup": (None, [_i, _i, _i, _p, _p, _p]),
            "oracle_calc_C": (_d, [_i, _p]),
            "oracle_build_Ndiag": (None, [_i, _i, _p, _p]),
            "oracle_interp_lookup": (_d, [_i, _i, _p, _d, _d, _i, _p, _p]),
            "oracle_lookup_A": (_i, [_i, _p, _p, _p, _i, _i, _i, _d, _d, _i, _p, _p]),
            "oracle_lookup_B": (_i, [_i, _i, _p, _p, _p, _p, _p, _i, _i, _i, _d, _d, _i, _p, _p]),
            "oracle_eigen_A": (_i, [_i, _p, _p, _p, _p]),
            "oracle_build_P": (None, [_i, _i, _p, _p, _p, _p]),
            "oracle_U_from_kappa": (_d, [_i, _p, _p, _d, _d]),
            "oracle_S_from_kappa": (_d, [_i, _p, _p, _p, _d]),
            "oracle_bisect_kappa": (None, [_i, _i, _i, _p, _p, _p, _d, _d, _d, _d, _d, _i, _p, _p, _p]),
            "oracle_build_T": (None, [_i, _i, _p, _p, _p, _p, _p]),
            "oracle_build_image": (None, [_i, _i, _p, _p, _p]),
            "oracle_build_U": (None, [_i, _i, _p, _p, _d, _p, _p]),
            "oracle_build_S": (None, [_i, _i, _p, _p, _p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _f64(a, shape=None):
    a = np.asarray(a, dtype=np.float64, order="F")
    if shape is not None:
        a = a.reshape(shape, order="F")
    return np.asfortranarray(a)


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def get_threads() -> int:
    return int(lib().oracle_get_threads())


def dlamch(c: str) -> float:
    return float(lib().oracle_dlamch(c.encode()))


def fft2d(a: np.ndarray, sign: int) -> np.ndarray:
    z = np.asfortranarray(np.array(a, dtype=np.complex128))
    lib().oracle_fft2d(z.shape[0], z.shape[1], int(sign), z.ctypes.data)
    return z


def polint(xa, ya, x):
    xa = _f64(xa)
    ya = _f64(ya)
    y = np.zeros(1)
    st = lib().oracle_polint(len(xa), _ptr(xa), _ptr(ya), float(x), _ptr(y))
    if st:
        raise ValueError("IMCOM ERROR: Two or more identical x input locations to IMCOM_POLINT")
    return float(y[0])


def rotate_image(im, theta_deg, npoly=7, conserve_flux=1):
    im = _f64(im)
    out = np.zeros_like(im, order="F")
    st = lib().oracle_rotate_image(im.shape[0], im.shape[1], _ptr(im), float(theta_deg),
                                   int(npoly), int(conserve_flux), _ptr(out))
    if st:
        raise ValueError("Neville trap in rotate_image")
    return out


def ft_r2c(F):
    F = _f64(F)
    Ft = np.zeros(F.shape, dtype=np.complex128, order="F")
    lib().oracle_ft_r2c(F.shape[0], F.shape[1], _ptr(F), _ptr(Ft))
    return Ft


def build_Alookup(Gt, npad=3):
    Gt = np.asfortranarray(Gt, dtype=np.complex128)
    nps, _, E = Gt.shape
    L = nps * npad
    out = np.zeros((L, L, E * (E + 1) // 2), order="F")
    lib().oracle_build_Alookup(nps, npad, E, _ptr(Gt), _ptr(out))
    return out


def build_Blookup(Gt, Gammat, npad=3):
    Gt = np.asfortranarray(Gt, dtype=np.complex128)
    Gammat = np.asfortranarray(Gammat, dtype=np.complex128)
    nps, _, E = Gt.shape
    L = nps * npad
    out = np.zeros((L, L, E), order="F")
    lib().oracle_build_Blookup(nps, npad, E, _ptr(Gt), _ptr(Gammat), _ptr(out))
    return out


def calc_C(Gammat):
    Gammat = np.asfortranarray(Gammat, dtype=np.complex128)
    return float(lib().oracle_calc_C(Gammat.shape[0], _ptr(Gammat)))


def build_Ndiag(n, noise):
    noise = _f64(noise)
    out = np.zeros(n)
    lib().oracle_build_Ndiag(int(n), len(noise), _ptr(noise), _ptr(out))
    return out


def interp_lookup(table, xarg, yarg, npoly=7):
    table = _f64(table)
    win = np.zeros(4, dtype=np.int32)
    st = np.zeros(1, dtype=np.int32)
    v = lib().oracle_interp_lookup(table.shape[0], table.shape[1], _ptr(table), float(xarg),
                                   float(yarg), int(npoly), _ptr(win), _ptr(st))
    return float(v), win, int(st[0])


def lookup_A(x_i, y_i, exp_i, psfconst, nps, npad, psfx, psfy, Alookup, npoly=7):
    x_i, y_i = _f64(x_i), _f64(y_i)
    exp_i = np.ascontiguousarray(exp_i, dtype=np.int32)
    n = len(x_i)
    A = np.zeros((n, n), order="F")
    st = lib().oracle_lookup_A(n, _ptr(x_i), _ptr(y_i), _ptr(exp_i), int(psfconst), int(nps),
                               int(npad), float(psfx), float(psfy), int(npoly),
                               _ptr(np.asfortranarray(Alookup)), _ptr(A))
    if st:
        raise ValueError("Neville trap in lookup_A")
    return A


def lookup_B(x_i, y_i, exp_i, X_a, Y_a, psfconst, nps, npad, psfx, psfy, Blookup, npoly=7):
    x_i, y_i, X_a, Y_a = _f64(x_i), _f64(y_i), _f64(X_a), _f64(Y_a)
    exp_i = np.ascontiguousarray(exp_i, dtype=np.int32)
    n, m = len(x_i), len(X_a)
    B = np.zeros((n, m), order="F")
    st = lib().oracle_lookup_B(n, m, _ptr(x_i), _ptr(y_i), _ptr(exp_i), _ptr(X_a), _ptr(Y_a),
                               int(psfconst), int(nps), int(npad), float(psfx), float(psfy),
                               int(npoly), _ptr(np.asfortranarray(Blookup)), _ptr(B))
    if st:
        raise ValueError("Neville trap in lookup_B")
    return B


def eigen_A(A):
    A = _f64(A)
    n = A.shape[0]
    Q = np.zeros((n, n), order="F")
    L = np.zeros(n)
    cond = np.zeros(1)
    info = lib().oracle_eigen_A(n, _ptr(A), _ptr(Q), _ptr(L), _ptr(cond))
    if info != 0:
        raise RuntimeError(f"IMCOM ERROR: DSYEVR info = {info}")
    return Q, L, float(cond[0])


def build_P(Q, B):
    Q, B = _f64(Q), _f64(B)
    n, m = B.shape
    P = np.zeros((n, m), order="F")
    P2 = np.zeros((n, m), order="F")
    lib().oracle_build_P(n, m, _ptr(Q), _ptr(B), _ptr(P), _ptr(P2))
    return P, P2


def U_from_kappa(L, P2a, C_a, k):
    L, P2a = _f64(L), _f64(P2a)
    return float(lib().oracle_U_from_kappa(len(L), _ptr(L), _ptr(P2a), float(C_a), float(k)))


def S_from_kappa(L, P2a, Ndiag, k):
    L, P2a, Ndiag = _f64(L), _f64(P2a), _f64(Ndiag)
    return float(lib().oracle_S_from_kappa(len(L), _ptr(L), _ptr(P2a), _ptr(Ndiag), float(k)))


def bisect_kappa(UnotS, L, P2, Ndiag, C_a, US, k_min, k_max, tol, maxnits):
    L, P2, Ndiag = _f64(L), _f64(P2), _f64(Ndiag)
    n, m = P2.shape
    K = np.zeros(m)
    US_out = np.zeros(m)
    nev = np.zeros(m, dtype=np.int32)
    lib().oracle_bisect_kappa(1 if UnotS else 0, n, m, _ptr(L), _ptr(P2), _ptr(Ndiag),
                              float(C_a), float(US), float(k_min), float(k_max), float(tol),
                              int(maxnits), _ptr(K), _ptr(US_out), _ptr(nev))
    return K, US_out, nev


def build_T(Q, P, L, K):
    Q, P, L, K = _f64(Q), _f64(P), _f64(L), _f64(K)
    n, m = P.shape
    T = np.zeros((n, m), order="F")
    lib().oracle_build_T(n, m, _ptr(Q), _ptr(P), _ptr(L), _ptr(K), _ptr(T))
    return T


def build_image(T, I):
    T, I = _f64(T), _f64(I)
    n, m = T.shape
    H = np.zeros(m)
    lib().oracle_build_image(n, m, _ptr(T), _ptr(I), _ptr(H))
    return H


def build_U(L, P2, C_a, K):
    L, P2, K = _f64(L), _f64(P2), _f64(K)
    n, m = P2.shape
    U = np.zeros(m)
    lib().oracle_build_U(n, m, _ptr(L), _ptr(P2), float(C_a), _ptr(K), _ptr(U))
    return U


def build_S(T, Ndiag):
    T, Ndiag = _f64(T), _f64(Ndiag)
    n, m = T.shape
    S = np.zeros(m)
    lib().oracle_build_S(n, m, _ptr(T), _ptr(Ndiag), _ptr(S))
    return S


@dataclass
class OracleResult:
    Gt: np.ndarray
    Gammat: np.ndarray
    C_a: float
    Alookup: np.ndarray
    Blookup: np.ndarray
    A: np.ndarray
    B: np.ndarray
    Q: np.ndarray
    L: np.ndarray
    condition: float
    P: np.ndarray
    P2: np.ndarray
    K: np.ndarray
    US: np.ndarray
    nevals: np.ndarray
    T: np.ndarray
    H: np.ndarray
    U: np.ndarray | None
    S: np.ndarray | None
    Ndiag: np.ndarray
    kappa_min: float
    kappa_max: float


def solve(prob, UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=53, npoly=7, npad=3,
          keep_tables=True) -> OracleResult:
    """Replay imcom.f90:90-169 (build branch) on a ``Problem`` (see
    imcom_b200.problem)."""
    E = prob.nexppsf
    nps = prob.nps
    pi = 3.141592653589793
    eps = dlamch("E")
    Gt = np.zeros((nps, nps, E), dtype=np.complex128, order="F")
    for e in range(E):
        G = prob.G_unrot[:, :, e]
        if abs(prob.rotangdeg[e]) > 2.0 * pi * eps:
            G = rotate_image(G, prob.rotangdeg[e], npoly, 1)
        Gt[:, :, e] = ft_r2c(G)
    Gammat = ft_r2c(prob.Gamma)
    Ndiag = build_Ndiag(prob.n, prob.noise)
    C_a = calc_C(Gammat)
    kmin, kmax = C_a * eps, C_a / eps
    Alookup = build_Alookup(Gt, npad)
    A = lookup_A(prob.x_i, prob.y_i, prob.exp_i, prob.psfconst, nps, npad, prob.psfxscale,
                 prob.psfyscale, Alookup, npoly)
    Q, L, cond = eigen_A(A)
    Blookup = build_Blookup(Gt, Gammat, npad)
    B = lookup_B(prob.x_i, prob.y_i, prob.exp_i, prob.X_a, prob.Y_a, prob.psfconst, nps, npad,
                 prob.psfxscale, prob.psfyscale, Blookup, npoly)
    P, P2 = build_P(Q, B)
    K, US, nev = bisect_kappa(UnotS, L, P2, Ndiag, C_a, US_max, kmin, kmax, US_tol, maxnits)
    T = build_T(Q, P, L, K)
    if UnotS:
        S = build_S(T, Ndiag)
        U = US
    else:
        U = build_U(L, P2, C_a, K)
        S = US
    H = build_image(T, prob.I_i)
    return OracleResult(Gt=Gt, Gammat=Gammat, C_a=C_a,
                        Alookup=Alookup if keep_tables else None,
                        Blookup=Blookup if keep_tables else None,
                        A=A, B=B, Q=Q, L=L, condition=cond, P=P, P2=P2, K=K, US=US,
                        nevals=nev, T=T, H=H, U=U, S=S, Ndiag=Ndiag,
                        kappa_min=kmin, kappa_max=kmax)
