"""Read a library device buffer into numpy through the CUDA runtime the
library itself loaded (test helper)."""
import ctypes as C

import numpy as np

_rt = None


def _cudart():
    global _rt
    if _rt is None:
        for name in ("libcudart.so.12", "libcudart.so"):
            try:
                _rt = C.CDLL(name)
                break
            except OSError:
                continue
        if _rt is None:
            raise OSError("CUDA runtime not found")
        _rt.cudaMemcpy2D.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_size_t,
                                     C.c_size_t, C.c_int]
        _rt.cudaMemcpy2D.restype = C.c_int
    return _rt


def download(solver, which: str, rows: int, cols: int) -> np.ndarray:
    """Column-major (rows, cols) float64 copy of buffer `which`."""
    solver.synchronize()
    ptr, ld = solver.device_buffer(which)
    out = np.zeros((rows, cols), order="F")
    st = _cudart().cudaMemcpy2D(out.ctypes.data, rows * 8, ptr, ld * 8, rows * 8, cols, 2)
    assert st == 0, f"cudaMemcpy2D failed ({st})"
    return out
