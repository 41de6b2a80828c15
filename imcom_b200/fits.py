"""FITS images without CFITSIO, through the library's C-ABI (host only).

The reference reads its inputs and reads and writes its cache and maps with
CFITSIO (imcom_io.f90:338-494).  These wrappers call the library's own
reader and writer (imcom_fits_size / _read / _write / _write_cube), which
need no GPU:

    from imcom_b200 import fits
    fits.write("A.fits", A)          # BITPIX -64, replaces an existing file
    A2 = fits.read("A.fits")         # any BITPIX; BSCALE/BZERO applied
    n1, n2, bitpix = fits.size("A.fits")

Arrays follow FITS (and Fortran) order: axis 1 is the first numpy axis of a
Fortran-ordered array.  Undefined pixels (NaN, or BLANK of integer images)
read as -666, the null value the reference asks CFITSIO for.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import ImcomError


def _call(name, *args):
    lib = _lib.load()
    st = getattr(lib, name)(*args)
    if st != 0:
        raise ImcomError(name, st, lib.imcom_fits_last_error().decode(errors="replace"))


def size(path: str) -> tuple[int, int, int]:
    """(NAXIS1, NAXIS2, BITPIX) of the primary image; NAXIS2 is 1 for a
    one-axis image."""
    n1, n2, bp = C.c_int(), C.c_int(), C.c_int()
    _call("imcom_fits_size", path.encode(), C.byref(n1), C.byref(n2), C.byref(bp))
    return n1.value, n2.value, bp.value


def read(path: str, shape: tuple[int, int] | None = None) -> np.ndarray:
    """The primary image as a Fortran-ordered float64 array of shape
    (NAXIS1, NAXIS2); `shape`, if given, must match the file."""
    n1, n2, _ = size(path) if shape is None else (shape[0], shape[1], 0)
    out = np.zeros((n1, n2), dtype=np.float64, order="F")
    _call("imcom_fits_read", path.encode(), int(n1), int(n2), C.c_void_p(out.ctypes.data))
    return out


def write(path: str, image) -> None:
    """Write a 2-D (or 1-D, as n x 1) image as BITPIX -64."""
    a = np.asarray(image, dtype=np.float64)
    if a.ndim == 1:
        a = a[:, None]
    if a.ndim != 2:
        raise ValueError("fits.write takes a 1-D or 2-D array; use write_cube for three axes")
    a = np.asfortranarray(a)
    _call("imcom_fits_write", path.encode(), int(a.shape[0]), int(a.shape[1]),
          C.c_void_p(a.ctypes.data))


def write_cube(path: str, cube) -> None:
    """Write a 3-D image as BITPIX -64 (axis 1 fastest)."""
    a = np.asfortranarray(np.asarray(cube, dtype=np.float64))
    if a.ndim != 3:
        raise ValueError("fits.write_cube takes a 3-D array")
    _call("imcom_fits_write_cube", path.encode(), int(a.shape[0]), int(a.shape[1]),
          int(a.shape[2]), C.c_void_p(a.ctypes.data))


def bench(n1: int = 8192, n2: int = 8192, path: str | None = None, reps: int = 3) -> dict:
    """Write and read throughput (GB/s of image data, best of `reps`) of an
    n1 x n2 BITPIX -64 image, beside a plain read of the same file's bytes
    into a new buffer (the bound for a reader that must also swap them)."""
    import os
    import tempfile
    import time

    a = np.asfortranarray(np.random.default_rng(0).standard_normal((n1, n2)))
    own = path is None
    if own:
        fd, path = tempfile.mkstemp(suffix=".fits")
        os.close(fd)

    def best(f):
        t = []
        for _ in range(reps):
            t0 = time.perf_counter()
            f()
            t.append(time.perf_counter() - t0)
        return a.nbytes / 1e9 / min(t)

    try:
        out = {"image": [n1, n2], "bytes": a.nbytes,
               "write_gbs": best(lambda: write(path, a)),
               "read_gbs": best(lambda: read(path)),
               "raw_read_gbs": best(lambda: np.fromfile(path, dtype=np.uint8))}
        if not np.array_equal(read(path), a):
            raise RuntimeError("FITS round trip differs")
    finally:
        if own:
            os.remove(path)
    out["read_frac_of_raw"] = out["read_gbs"] / out["raw_read_gbs"]
    return out


__all__ = ["size", "read", "write", "write_cube", "bench"]


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="FITS read/write throughput of the library")
    ap.add_argument("--bench", nargs=2, type=int, metavar=("N1", "N2"), default=[8192, 8192])
    ap.add_argument("--path", default=None, help="file to use (default: a temporary file)")
    args = ap.parse_args()
    print(json.dumps(bench(*args.bench, path=args.path)))
