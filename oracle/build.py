"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/imcom_oracle.cpp`` into ``oracle/libimcom_oracle.so`` with
OpenMP, linking the LAPACK/BLAS that scipy bundles (``libscipy_openblas``).
The reference Fortran itself cannot be compiled in this environment (no
Fortran compiler, FFTW or CFITSIO), so there is no ``oracle/_ref`` build.

Usage: ``python oracle/build.py`` (also called by ``__graft_entry__.build``).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "imcom_oracle.cpp")
OUT = os.path.join(HERE, "libimcom_oracle.so")


def openblas_path() -> str:
    import scipy

    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError("scipy's bundled OpenBLAS not found in " + libdir)
    return cands[0]


def build(force: bool = False, verbose: bool = False) -> str:
    if (not force and os.path.exists(OUT)
            and os.path.getmtime(OUT) >= os.path.getmtime(SRC)
            and os.path.getmtime(OUT) >= os.path.getmtime(__file__)):
        return OUT
    blas = openblas_path()
    cmd = [
        "g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
        SRC, "-o", OUT + ".tmp",
        "-L" + os.path.dirname(blas), "-l:" + os.path.basename(blas),
        "-Wl,-rpath," + os.path.dirname(blas),
    ]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
