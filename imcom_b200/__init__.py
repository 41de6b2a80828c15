"""imcom_b200: the IMCOM solve path on one B200 (sm_100a).

The compute lives in ``libimcom_gpu.so`` (hand-written CUDA behind the C-ABI of
``include/imcom_gpu.h``).  This package holds the ctypes binding
(``_lib``), a host-side mirror of the reference's solve-path routines
(``api.Solver``), the problem model (``problem``), the seeded synthetic
inputs (``synth``), FITS images without CFITSIO (``fits``), the many-patch
driver (``batch``, ``replicas``), the learned-kappa model (``kappa_model``)
measurements that print one JSON line (``t_reuse``, ``table_fft``) and the
stage-by-stage timer (``stages``).
"""
from .api import (EIGH_DC, EIGH_JACOBI, EIGH_LIBRARY, EIGH_TWOSTAGE, EPS,  # noqa: F401
                  ImcomError, SolveResult, Solver)

__all__ = ["Solver", "SolveResult", "ImcomError", "EIGH_DC", "EIGH_JACOBI", "EIGH_LIBRARY",
           "EIGH_TWOSTAGE", "EPS"]
