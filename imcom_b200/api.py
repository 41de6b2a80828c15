"""Host-side mirror of the reference's solve-path interface over the C-ABI.

``Solver`` wraps one ``imcom_ctx``.  Its methods follow the reference's
routines one for one (imcom_get_A / imcom_get_QL / imcom_get_B / imcom_get_P /
imcom_get_T / imcom_build_image, imcom_matrix.f90 and imcom_bisect.f90) and
take/return numpy arrays in the reference's Fortran layout.  ``solve`` replays
the build branch of the driver (imcom.f90:90-169).

Every call goes through ``libimcom_gpu.so``; a non-zero status raises
``ImcomError`` with the library's message (the reference's `write + stop`).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import ImcomError

EIGH_DC, EIGH_JACOBI, EIGH_LIBRARY, EIGH_TWOSTAGE = 0, 1, 2, 3
OPT_EIGENSOLVER, OPT_EIGEN_MAXITER = 1, 2
OPT_DC_MAXITER, OPT_STALL_TEST = 15, 16
STALL_SPLIT, STALL_TRIDIAG = 1, 2
OPT_PRECISION, OPT_SPLIT_SLICES_P, OPT_SPLIT_SLICES_T = 3, 4, 5
OPT_SPLIT_TOL_US, OPT_SPLIT_TOL_T = 6, 7
PREC_FP64, PREC_SPLIT = 0, 1
OPT_BISECT_KERNEL = 8
BISECT_AUTO, BISECT_STREAM, BISECT_RESIDENT = 0, 1, 2
OPT_BISECT_CTAS_PER_SM = 9
OPT_SM_SHARE = 10
OPT_TAIL_CTAS = 11
OPT_STACK_KERNEL = 12
STACKS_GEMM, STACKS_STREAM, STACKS_AUTO = 0, 1, 2
OPT_TABLE_FFT = 13
OPT_KAPPA_FEATURES = 14
OPT_KAPPA_START = 17
TABLE_FFT_CUFFT, TABLE_FFT_OWN, TABLE_FFT_AUTO = 0, 1, 2
SPLIT_INFO = ("slices_P", "slices_T", "fp64_pixels_P", "fp64_columns_T", "max_bound_US",
              "max_bound_T_from_P", "max_bound_T_product", "P_split")
STAGES = ("spectra", "build_A", "eigen_A", "build_B", "build_P", "bisect", "build_T", "epilogue",
          "eig_tridiag", "eig_dc", "eig_backtransform")
EPS = 1.1102230246251565e-16  # DLAMCH('Epsilon')


def _f64(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _ptr(a):
    return None if a is None else a.ctypes.data


class Solver:
    """One GPU context holding the solve path's module state."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        st = self.lib.imcom_gpu_create(int(device), C.byref(h))
        if st != 0:
            raise ImcomError("imcom_gpu_create", st, "no usable CUDA device")
        self.h = h
        self.n = self.m = 0
        self.C_a = None

    # -- plumbing ---------------------------------------------------------
    def _call(self, name, *args):
        st = getattr(self.lib, name)(self.h, *args)
        if st != 0:
            msg = self.lib.imcom_gpu_last_error(self.h)
            raise ImcomError(name, st, msg.decode() if msg else "")
        return st

    def close(self):
        if getattr(self, "h", None):
            self.lib.imcom_gpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        self._call("imcom_gpu_synchronize")

    def set_option(self, option: int, value: int):
        self._call("imcom_gpu_set_option", int(option), int(value))

    def set_eigensolver(self, mode: int):
        self.set_option(OPT_EIGENSOLVER, mode)

    def set_precision(self, split: bool, slices_P: int = 7, slices_T: int = 6,
                      tol_us_exp: int = 7, tol_t_exp: int = 8):
        """FP64 (split=False) or the audited int8 split product for P and T."""
        self.set_option(OPT_PRECISION, PREC_SPLIT if split else PREC_FP64)
        self.set_option(OPT_SPLIT_SLICES_P, slices_P)
        self.set_option(OPT_SPLIT_SLICES_T, slices_T)
        self.set_option(OPT_SPLIT_TOL_US, tol_us_exp)
        self.set_option(OPT_SPLIT_TOL_T, tol_t_exp)

    def split_pixels(self):
        """(fp64_P, fp64_T): per-pixel flags of the audit's FP64 recomputations."""
        fp = np.zeros(self.m, dtype=np.int32)
        ft = np.zeros(self.m, dtype=np.int32)
        self._call("imcom_gpu_split_pixels", _ptr(fp), _ptr(ft))
        return fp.astype(bool), ft.astype(bool)

    def split_info(self) -> dict:
        v = np.zeros(8)
        self._call("imcom_gpu_split_info", _ptr(v))
        return dict(zip(SPLIT_INFO, v.tolist()))

    def stage_times(self) -> dict:
        ms = np.zeros(len(STAGES))
        self._call("imcom_gpu_stage_times", _ptr(ms))
        return dict(zip(STAGES, ms.tolist()))

    def table_times(self) -> dict:
        """Milliseconds of the last A and B lookup-table builds."""
        ms = np.zeros(2)
        self._call("imcom_gpu_table_times", _ptr(ms))
        return {"A_tables": float(ms[0]), "B_tables": float(ms[1])}

    def stream(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        self._call("imcom_gpu_get_stream", C.byref(s))
        return s.value

    def launch_count(self) -> int:
        """This library's kernel launches so far (process-wide)."""
        v = C.c_longlong()
        self._call("imcom_gpu_launch_count", C.byref(v))
        return int(v.value)

    def eigh_jacobi_batched(self, A):
        """Eigendecomposition of a stack of small symmetric positive
        semi-definite matrices A (count, n, n), n <= 112, one thread block each
        (one-sided Jacobi).  Returns Q (count, n, n) with eigenvectors in
        columns, L (count, n) and the sweeps used, ascending per matrix."""
        A = np.asarray(A, dtype=np.float64)
        if A.ndim == 2:
            A = A[None]
        count, n = A.shape[0], A.shape[1]
        At = np.ascontiguousarray(np.transpose(A, (0, 2, 1)))  # column-major per matrix
        Q = np.zeros_like(At)
        L = np.zeros((count, n))
        sw = np.zeros(count, dtype=np.int32)
        self._call("imcom_gpu_eigh_jacobi_batched", int(n), int(count), _ptr(At), _ptr(Q), _ptr(L),
                   _ptr(sw))
        return np.transpose(Q, (0, 2, 1)), L, sw

    def device_buffer(self, which: str):
        p, ld = C.c_void_p(), C.c_longlong()
        self._call("imcom_gpu_device_buffer", which.encode(), C.byref(p), C.byref(ld))
        return p.value, ld.value

    # -- module state -----------------------------------------------------
    def set_inputs(self, x_i, y_i, exp_i, X_a, Y_a, I_i=None, Ndiag=None, psfxscale=1.0,
                   psfyscale=1.0):
        x_i, y_i, X_a, Y_a = _f64(x_i), _f64(y_i), _f64(X_a), _f64(Y_a)
        I_i = None if I_i is None else _f64(I_i)
        Ndiag = None if Ndiag is None else _f64(Ndiag)
        exp_i = np.ascontiguousarray(exp_i, dtype=np.int32)
        self.n, self.m = len(x_i), len(X_a)
        self._keep = (x_i, y_i, X_a, Y_a, I_i, Ndiag, exp_i)
        self._call("imcom_gpu_set_inputs", self.n, self.m, _ptr(x_i), _ptr(y_i), _ptr(exp_i),
                   _ptr(X_a), _ptr(Y_a), _ptr(I_i), _ptr(Ndiag), float(psfxscale),
                   float(psfyscale))

    def set_psfs(self, G_unrot, rotangdeg, Gamma, psfconst):
        G = _f64(G_unrot)
        if G.ndim == 2:
            G = G[:, :, None]
        G = np.asfortranarray(G)
        rot = _f64(rotangdeg)
        Gam = _f64(Gamma)
        nps, E = G.shape[0], G.shape[2]
        self._call("imcom_gpu_set_psfs", nps, E, int(psfconst), _ptr(G), _ptr(rot[:E].copy()),
                   _ptr(Gam))
        self.nps, self.nexppsf = nps, E

    def set_problem(self, prob):
        from .problem import build_Ndiag
        self.set_inputs(prob.x_i, prob.y_i, prob.exp_i, prob.X_a, prob.Y_a, prob.I_i,
                        build_Ndiag(prob.n, prob.noise), prob.psfxscale, prob.psfyscale)
        self.set_psfs(prob.G_unrot, prob.rotangdeg, prob.Gamma, prob.psfconst)

    # -- solve path (reference routine names) --------------------------------
    def psf_spectra(self, npoly=7, spectra=False):
        Cout = np.zeros(1)
        Gt = Gm = None
        if spectra:
            Gt = np.zeros((self.nps, self.nps, self.nexppsf), dtype=np.complex128, order="F")
            Gm = np.zeros((self.nps, self.nps), dtype=np.complex128, order="F")
        self._call("imcom_gpu_psf_spectra", int(npoly), _ptr(Cout), _ptr(Gt), _ptr(Gm))
        self.C_a = float(Cout[0])
        return (self.C_a, Gt, Gm) if spectra else self.C_a

    def build_A(self, npoly=7, npad=3, out=True):
        A = np.zeros((self.n, self.n), order="F") if out else None
        self._call("imcom_gpu_build_A", int(npoly), int(npad), _ptr(A))
        return A

    def load_A(self, A):
        self._call("imcom_gpu_load_A", _ptr(_f64(A)))

    def eigen_A(self, out=True):
        Q = np.zeros((self.n, self.n), order="F") if out else None
        L = np.zeros(self.n)
        cond = np.zeros(1)
        self._call("imcom_gpu_eigen_A", _ptr(Q), _ptr(L), _ptr(cond))
        return Q, L, float(cond[0])

    def load_QL(self, Q, L):
        self._call("imcom_gpu_load_QL", _ptr(_f64(Q)), _ptr(_f64(L)))

    def build_B(self, npoly=7, npad=3, out=True):
        B = np.zeros((self.n, self.m), order="F") if out else None
        self._call("imcom_gpu_build_B", int(npoly), int(npad), _ptr(B))
        return B

    def load_B(self, B):
        self._call("imcom_gpu_load_B", _ptr(_f64(B)))

    def build_P(self, out=True):
        P = np.zeros((self.n, self.m), order="F") if out else None
        self._call("imcom_gpu_build_P", _ptr(P))
        return P

    def load_P(self, P):
        self._call("imcom_gpu_load_P", _ptr(_f64(P)))

    def free_AB(self):
        self._call("imcom_gpu_free_AB")

    def bisect_kappa(self, UnotS, US_max, k_min, k_max, tol, maxnits, C_a=None, out=True):
        C_a = self.C_a if C_a is None else C_a
        K = np.zeros(self.m) if out else None
        US = np.zeros(self.m) if out else None
        nev = np.zeros(self.m, dtype=np.int32) if out else None
        self._call("imcom_gpu_bisect_kappa", 1 if UnotS else 0, float(US_max), float(k_min),
                   float(k_max), float(tol), int(maxnits), float(C_a), _ptr(K), _ptr(US),
                   _ptr(nev))
        return K, US, nev

    def bisect_kappa_learned(self, UnotS, US_max, k_min, k_max, tol, maxnits, C_a=None,
                             out=True):
        C_a = self.C_a if C_a is None else C_a
        K = np.zeros(self.m) if out else None
        US = np.zeros(self.m) if out else None
        nev = np.zeros(self.m, dtype=np.int32) if out else None
        fb = np.zeros(self.m, dtype=np.int32) if out else None
        self._call("imcom_gpu_bisect_kappa_learned", 1 if UnotS else 0, float(US_max),
                   float(k_min), float(k_max), float(tol), int(maxnits), float(C_a), _ptr(K),
                   _ptr(US), _ptr(nev), _ptr(fb))
        return K, US, nev, fb

    def build_T(self, out=True):
        T = np.zeros((self.n, self.m), order="F") if out else None
        self._call("imcom_gpu_build_T", _ptr(T))
        return T

    def load_T(self, T):
        self._call("imcom_gpu_load_T", _ptr(_f64(T)))

    def load_K(self, K):
        self._call("imcom_gpu_load_K", _ptr(_f64(K)))

    def build_image(self, out=True):
        H = np.zeros(self.m) if out else None
        self._call("imcom_gpu_build_image", _ptr(H))
        return H

    def build_images(self, I_stack, out=True):
        """H = T^T I for image stacks sharing the resident T's geometry:
        I_stack is (n, stacks) (or (n,) for one), H is (m, stacks)."""
        I = _f64(I_stack)
        if I.ndim == 1:
            I = I[:, None]
        if I.ndim != 2 or I.shape[0] != self.n:
            raise ValueError(f"I_stack must have {self.n} rows (one per input pixel)")
        I = np.asfortranarray(I)
        H = np.zeros((self.m, I.shape[1]), order="F") if out else None
        self._call("imcom_gpu_build_images", int(I.shape[1]), _ptr(I), _ptr(H))
        return H

    def build_images_device(self, dI, dH):
        """The same on torch CUDA tensors (column-major: dI of shape
        (stacks, n), dH (stacks, m), each row a stack), ordered on the library
        stream and not synchronised."""
        if dI.dim() != 2 or dI.shape[1] != self.n or dH.shape != (dI.shape[0], self.m):
            raise ValueError("dI must be (stacks, n) and dH (stacks, m)")
        if dI.stride(1) != 1 or dH.stride(1) != 1:
            raise ValueError("dI and dH need unit stride along the pixels")
        # a single stack has no second row, so its row stride is arbitrary
        # (numpy and torch may give a length-1 axis any stride)
        one = dI.shape[0] == 1
        ldi = self.n if one else int(dI.stride(0))
        ldh = self.m if one else int(dH.stride(0))
        self._call("imcom_gpu_build_images_device", int(dI.shape[0]), dI.data_ptr(), ldi,
                   dH.data_ptr(), ldh)

    def build_S(self, out=True):
        S = np.zeros(self.m) if out else None
        self._call("imcom_gpu_build_S", _ptr(S))
        return S

    def build_U(self, C_a=None, out=True):
        C_a = self.C_a if C_a is None else C_a
        U = np.zeros(self.m) if out else None
        self._call("imcom_gpu_build_U", float(C_a), _ptr(U))
        return U

    def kappa_features(self, UnotS, US_max, C_a=None):
        C_a = self.C_a if C_a is None else C_a
        F = np.zeros((12, self.m), dtype=np.float32)  # feature-major: F[k, a] at k * m + a
        self._call("imcom_gpu_kappa_features", 1 if UnotS else 0, float(US_max), float(C_a),
                   _ptr(F))
        return F

    def mlp_train(self, feat, target, params, epochs=30, batch=512, lr=2e-3, seed=1):
        """Train on the GPU (Adam); feat (12, N) and target (N) normalised."""
        feat = np.ascontiguousarray(feat, dtype=np.float32)  # feature-major
        target = np.ascontiguousarray(target, dtype=np.float32)
        p = np.ascontiguousarray(params, dtype=np.float32).copy()
        loss = np.zeros(epochs, dtype=np.float32)
        self._call("imcom_gpu_mlp_train", int(target.size), _ptr(feat), _ptr(target), int(epochs),
                   int(batch), C.c_float(lr), C.c_uint(seed), _ptr(p), _ptr(loss))
        return p, loss

    def mlp_gradient(self, feat, target, params):
        feat = np.ascontiguousarray(feat, dtype=np.float32)  # feature-major
        target = np.ascontiguousarray(target, dtype=np.float32)
        p = np.ascontiguousarray(params, dtype=np.float32)
        g = np.zeros_like(p)
        loss = np.zeros(1, dtype=np.float32)
        self._call("imcom_gpu_mlp_gradient", int(target.size), _ptr(feat), _ptr(target), _ptr(p),
                   _ptr(g), _ptr(loss))
        return g, float(loss[0])

    def mlp_set_weights(self, W1, b1, W2, b2, W3, b3, mean, std):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (W1, b1, W2, b2, W3, b3, mean, std)]
        self._call("imcom_gpu_mlp_set_weights", *[_ptr(a) for a in arrs])

    # -- whole solve --------------------------------------------------------
    def solve(self, prob, UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=53, npoly=7, npad=3,
              learned=False, outputs=True, keep=("A", "B", "Q", "P", "T")):
        """Replay imcom.f90:90-169: spectra, A, QL, B, P, kappa, T, U/S, H."""
        self.set_problem(prob)
        C_a = self.psf_spectra(npoly)
        kmin, kmax = C_a * EPS, C_a / EPS
        res = SolveResult(C_a=C_a, kappa_min=kmin, kappa_max=kmax)
        res.A = self.build_A(npoly, npad, out=outputs and "A" in keep)
        res.Q, res.L, res.condition = self.eigen_A(out=outputs and "Q" in keep)
        res.B = self.build_B(npoly, npad, out=outputs and "B" in keep)
        res.P = self.build_P(out=outputs and "P" in keep)
        if learned:
            res.K, res.US, res.nevals, res.fallback = self.bisect_kappa_learned(
                UnotS, US_max, kmin, kmax, US_tol, maxnits, C_a)
        else:
            res.K, res.US, res.nevals = self.bisect_kappa(UnotS, US_max, kmin, kmax, US_tol,
                                                          maxnits, C_a)
        res.T = self.build_T(out=outputs and "T" in keep)
        if UnotS:
            res.U = res.US
            res.S = self.build_S()
        else:
            res.S = res.US
            res.U = self.build_U(C_a)
        res.H = self.build_image()
        return res


@dataclass
class SolveResult:
    C_a: float = 0.0
    kappa_min: float = 0.0
    kappa_max: float = 0.0
    A: np.ndarray | None = None
    B: np.ndarray | None = None
    Q: np.ndarray | None = None
    L: np.ndarray | None = None
    condition: float = 0.0
    P: np.ndarray | None = None
    K: np.ndarray | None = None
    US: np.ndarray | None = None
    nevals: np.ndarray | None = None
    fallback: np.ndarray | None = None
    T: np.ndarray | None = None
    U: np.ndarray | None = None
    S: np.ndarray | None = None
    H: np.ndarray | None = None
