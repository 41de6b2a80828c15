"""Independent numpy/scipy restatement of the IMCOM solve path (small cases).

A second oracle written separately from oracle/imcom_oracle.cpp: pure-Python
Neville (imcom_proc.f90:351-429), numpy FFTs with np.roll for Fortran CSHIFT
(imcom_matrix.f90:361-493), scipy's LAPACK DSYEVR driver (eigh(driver="evr"),
imcom_matrix.f90:617-643), numpy products for P and T, and the bisection
of imcom_bisect.f90:174-267 in plain Python.  Used only by
make_golden.py to produce the committed fixtures that pin the C++ oracle.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg

EPS = float(np.finfo(np.float64).eps / 2)  # DLAMCH('E')
PI = 3.141592653589793


def polint(xa, ya, x):
    n = len(xa)
    c = list(ya)
    d = list(ya)
    ho = [xa[i] - x for i in range(n)]
    dif = [abs(x - xa[i]) for i in range(n)]
    ns = int(np.argmin(dif)) + 1
    y = ya[ns - 1]
    ns -= 1
    for m in range(1, n):
        den = [ho[i] - ho[i + m] for i in range(n - m)]
        if any(abs(v) <= EPS for v in den):
            raise ValueError("duplicate abscissae")
        den = [(c[i + 1] - d[i]) / den[i] for i in range(n - m)]
        for i in range(n - m):
            d[i] = ho[i + m] * den[i]
            c[i] = ho[i] * den[i]
        if 2 * ns < n - m:
            dy = c[ns]
        else:
            dy = d[ns - 1]
            ns -= 1
        y = y + dy
    return y


def polin2(x1a, x2a, ya, x1, x2):
    ym = [polint(x2a, list(ya[j, :]), x2) for j in range(len(x1a))]
    return polint(x1a, ym, x1)


def interp_lookup(tab, xarg, yarg, npm=3):
    n1, n2 = tab.shape
    iarg = float(n1 // 2 + 1) + xarg
    jarg = float(n2 // 2 + 1) + yarg
    fi, fj, ci, cj = math.floor(iarg), math.floor(jarg), math.ceil(iarg), math.ceil(jarg)
    if fi >= 1 and fj >= 1 and ci <= n1 and cj <= n2:
        imin, jmin = max(1, fi - npm), max(1, fj - npm)
        imax, jmax = min(n1, ci + npm), min(n2, cj + npm)
        return polin2([float(i) for i in range(imin, imax + 1)],
                      [float(j) for j in range(jmin, jmax + 1)],
                      tab[imin - 1:imax, jmin - 1:jmax], iarg, jarg)
    return 0.0


def rotate_image(im, theta_deg, npm=3):
    nim1, nim2 = im.shape
    th = math.fmod(theta_deg, 360.0) * PI / 180.0
    cost, sint = math.cos(th), math.sin(th)
    xc, yc = (nim1 + 1) / 2.0, (nim2 + 1) / 2.0
    out = np.zeros_like(im)
    for iout in range(1, nim1 + 1):
        xout = iout - xc
        for jout in range(1, nim2 + 1):
            yout = jout - yc
            xs = xout * cost + yout * sint + xc
            ys = -xout * sint + yout * cost + yc
            fi, fj, ci, cj = math.floor(xs), math.floor(ys), math.ceil(xs), math.ceil(ys)
            if fi >= 1 and fj >= 1 and ci <= nim1 and cj <= nim2:
                imin, jmin = max(1, fi - npm), max(1, fj - npm)
                imax, jmax = min(nim1, ci + npm), min(nim2, cj + npm)
                out[iout - 1, jout - 1] = polin2(
                    [float(i) for i in range(imin, imax + 1)],
                    [float(j) for j in range(jmin, jmax + 1)],
                    im[imin - 1:imax, jmin - 1:jmax], xs, ys)
    return im.sum() * out / out.sum()


def ft_r2c(F):
    return np.fft.fft2(F)


def cshift(X, s, axis):
    return np.roll(X, -s, axis=axis)


def build_lookup(Gt, Gammat=None, npad=3):
    nps = Gt.shape[0]
    E = Gt.shape[2]
    L = nps * npad
    n0 = (L - nps) // 2
    tabs = []
    jobs = ([(e, f) for e in range(E) for f in range(e, E)] if Gammat is None
            else [(e, None) for e in range(E)])
    out = np.zeros((L, L, len(jobs)), order="F")
    for (e, f) in jobs:
        if Gammat is None:
            X = np.conj(Gt[:, :, e]) * Gt[:, :, f]
            ial = (e + 1) + (f + 1) * f // 2
        else:
            X = np.conj(Gammat) * Gt[:, :, e]
            ial = e + 1
        u = np.zeros((L, L), dtype=complex)
        u[n0:n0 + nps, n0:n0 + nps] = cshift(cshift(X, nps // 2, 1), nps // 2, 0)
        u = cshift(cshift(u, L // 2, 1), L // 2, 0)
        tmp = np.fft.ifft2(u) * (L * L)
        t = cshift(cshift(np.real(tmp), L // 2, 1), L // 2, 0)
        if Gammat is not None:
            t = -2.0 * t
        out[:, :, ial - 1] = t / nps / nps
    return out


def lookup_A(prob, Alookup, npad=3):
    n = prob.n
    A = np.zeros((n, n), order="F")
    for i in range(n):
        for j in range(i, n):
            ial = 1 if prob.psfconst else prob.exp_i[i] + prob.exp_i[j] * (prob.exp_i[j] - 1) // 2
            dx = npad * (prob.x_i[j] - prob.x_i[i]) / prob.psfxscale
            dy = npad * (prob.y_i[j] - prob.y_i[i]) / prob.psfyscale
            A[i, j] = interp_lookup(Alookup[:, :, ial - 1], dx, dy)
    iu = np.triu_indices(n, 1)
    A[(iu[1], iu[0])] = A[iu]
    return A


def lookup_B(prob, Blookup, npad=3):
    n, m = prob.n, prob.m
    B = np.zeros((n, m), order="F")
    for i in range(n):
        t = 1 if prob.psfconst else prob.exp_i[i]
        for a in range(m):
            dx = npad * (prob.x_i[i] - prob.X_a[a]) / prob.psfxscale
            dy = npad * (prob.y_i[i] - prob.Y_a[a]) / prob.psfyscale
            B[i, a] = interp_lookup(Blookup[:, :, t - 1], dx, dy)
    return B


def U_from_kappa(L, P2a, C, k):
    return (C - np.sum((L + 2.0 * k) * P2a / ((L + k) * (L + k))) / 4.0) / C


def S_from_kappa(L, P2a, Nd, k):
    return np.sum(Nd * P2a / ((L + k) * (L + k))) / 4.0


def bisect(UnotS, L, P2, Nd, C, US, kmin, kmax, tol, maxnits):
    m = P2.shape[1]
    K = np.zeros(m)
    out = np.zeros(m)
    nev = np.zeros(m, dtype=np.int32)
    for a in range(m):
        f_of = ((lambda k: U_from_kappa(L, P2[:, a], C, k)) if UnotS
                else (lambda k: S_from_kappa(L, P2[:, a], Nd, k)))
        k0, k1 = (kmin, kmax) if UnotS else (kmax, kmin)
        v = f_of(k0)
        ne = 1
        if v - US < 0.0:
            root = math.log10(k0)
            dx = math.log10(k1) - root
            for _ in range(maxnits):
                dx = 0.5 * dx
                mid = root + dx
                fmid = f_of(10.0 ** mid) - US
                ne += 1
                if fmid < 0.0:
                    root = mid
                    v = fmid + US
                    if abs(fmid) < tol:
                        break
                if abs(fmid) < C * EPS:
                    break
            K[a] = 10.0 ** root
        else:
            K[a] = k0
        out[a] = v
        nev[a] = ne
    return K, out, nev


def solve(prob, UnotS=True, US=1e-6, tol=1e-8, maxnits=53):
    from imcom_b200.problem import build_Ndiag
    E = prob.nexppsf
    Gt = np.zeros((prob.nps, prob.nps, E), dtype=complex, order="F")
    for e in range(E):
        G = prob.G_unrot[:, :, e]
        if abs(prob.rotangdeg[e]) > 2.0 * PI * EPS:
            G = rotate_image(G, prob.rotangdeg[e])
        Gt[:, :, e] = ft_r2c(G)
    Gammat = ft_r2c(prob.Gamma)
    C = float(np.sum(np.real(Gammat * np.conj(Gammat)))) / prob.nps / prob.nps
    kmin, kmax = C * EPS, C / EPS
    A = lookup_A(prob, build_lookup(Gt))
    w, V = scipy.linalg.eigh(A, driver="evr")
    L = w[::-1].copy()
    Q = np.asfortranarray(V[:, ::-1])
    B = lookup_B(prob, build_lookup(Gt, Gammat))
    P = Q.T @ B
    P2 = P * P
    Nd = build_Ndiag(prob.n, prob.noise)
    K, US_a, nev = bisect(UnotS, L, P2, Nd, C, US, kmin, kmax, tol, maxnits)
    T = -(Q @ (P / (L[:, None] + K[None, :]))) / 2.0
    H = T.T @ prob.I_i
    S = np.sum(T * (T * Nd[:, None]), axis=0)
    U = np.array([U_from_kappa(L, P2[:, a], C, K[a]) for a in range(prob.m)])
    return dict(Gt=Gt, Gammat=Gammat, C=C, A=A, B=B, L=L, Q=Q, P=P, K=K, US=US_a, nevals=nev,
                T=T, H=H, S=S, U=U, kappa_min=kmin, kappa_max=kmax)
