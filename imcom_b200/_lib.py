"""ctypes binding of ``libimcom_gpu.so`` (the C-ABI declared in include/imcom_gpu.h).

There is no CPU fallback: importing the library fails loudly when the shared
object has not been built, and every call raises ``ImcomError`` on a non-zero
status.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libimcom_gpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "imcom_gpu.h")

_d, _i, _p, _ll = C.c_double, C.c_int, C.c_void_p, C.c_longlong

# name -> (restype, argtypes)
SIGNATURES = {
    "imcom_gpu_create": (_i, [_i, C.POINTER(_p)]),
    "imcom_gpu_destroy": (_i, [_p]),
    "imcom_gpu_last_error": (C.c_char_p, [_p]),
    "imcom_gpu_synchronize": (_i, [_p]),
    "imcom_gpu_set_option": (_i, [_p, _i, _ll]),
    "imcom_gpu_set_inputs": (_i, [_p, _i, _i, _p, _p, _p, _p, _p, _p, _p, _d, _d]),
    "imcom_gpu_set_psfs": (_i, [_p, _i, _i, _i, _p, _p, _p]),
    "imcom_gpu_psf_spectra": (_i, [_p, _i, _p, _p, _p]),
    "imcom_gpu_build_A": (_i, [_p, _i, _i, _p]),
    "imcom_gpu_load_A": (_i, [_p, _p]),
    "imcom_gpu_eigen_A": (_i, [_p, _p, _p, _p]),
    "imcom_gpu_load_QL": (_i, [_p, _p, _p]),
    "imcom_gpu_build_B": (_i, [_p, _i, _i, _p]),
    "imcom_gpu_load_B": (_i, [_p, _p]),
    "imcom_gpu_build_P": (_i, [_p, _p]),
    "imcom_gpu_load_P": (_i, [_p, _p]),
    "imcom_gpu_free_AB": (_i, [_p]),
    "imcom_gpu_bisect_kappa": (_i, [_p, _i, _d, _d, _d, _d, _i, _d, _p, _p, _p]),
    "imcom_gpu_bisect_kappa_learned": (_i, [_p, _i, _d, _d, _d, _d, _i, _d, _p, _p, _p, _p]),
    "imcom_gpu_build_T": (_i, [_p, _p]),
    "imcom_gpu_load_T": (_i, [_p, _p]),
    "imcom_gpu_load_K": (_i, [_p, _p]),
    "imcom_gpu_build_image": (_i, [_p, _p]),
    "imcom_gpu_build_images": (_i, [_p, _i, _p, _p]),
    "imcom_gpu_build_images_device": (_i, [_p, _i, _p, _ll, _p, _ll]),
    "imcom_gpu_build_S": (_i, [_p, _p]),
    "imcom_gpu_build_U": (_i, [_p, _d, _p]),
    "imcom_gpu_kappa_features": (_i, [_p, _i, _d, _d, _p]),
    "imcom_gpu_mlp_set_weights": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "imcom_gpu_mlp_train": (_i, [_p, _i, _p, _p, _i, _i, C.c_float, C.c_uint, _p, _p]),
    "imcom_gpu_mlp_gradient": (_i, [_p, _i, _p, _p, _p, _p, _p]),
    "imcom_gpu_split_info": (_i, [_p, _p]),
    "imcom_gpu_split_pixels": (_i, [_p, _p, _p]),
    "imcom_gpu_build_P_noalloc": (_i, [_p, _ll, _p, _ll, _p, _ll, _i, _i, _p]),
    "imcom_gpu_eigh_jacobi_batched": (_i, [_p, _i, _i, _p, _p, _p, _p]),
    "imcom_gpu_band_reduce": (_i, [_p, _p, _i]),
    "imcom_fits_size": (_i, [C.c_char_p, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "imcom_fits_read": (_i, [C.c_char_p, _i, _i, _p]),
    "imcom_fits_write": (_i, [C.c_char_p, _i, _i, _p]),
    "imcom_fits_write_cube": (_i, [C.c_char_p, _i, _i, _i, _p]),
    "imcom_fits_last_error": (C.c_char_p, []),
    "imcom_gpu_device_buffer": (_i, [_p, C.c_char, C.POINTER(_p), C.POINTER(_ll)]),
    "imcom_gpu_get_stream": (_i, [_p, C.POINTER(_p)]),
    "imcom_gpu_launch_count": (_i, [_p, C.POINTER(_ll)]),
    "imcom_gpu_stage_times": (_i, [_p, _p]),
    "imcom_gpu_table_times": (_i, [_p, _p]),
}


def header_symbols() -> list[str]:
    """Function names declared in include/imcom_gpu.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(imcom_(?:gpu|fits)_\w+)\s*\(", txt)))


class ImcomError(RuntimeError):
    def __init__(self, fn, status, msg):
        super().__init__(f"{fn} returned {status}: {msg}")
        self.status = status


_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m imcom_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib
