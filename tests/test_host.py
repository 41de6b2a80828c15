"""Host-side logic restated from imcom_io / imcom_proc, and the C-ABI
library's exports (no GPU calls)."""
import ctypes
import os

import numpy as np
import pytest

from imcom_b200 import problem, synth, _lib


def test_mask_images_exposure_major():
    im = np.arange(2 * 3 * 2, dtype=float).reshape((2, 3, 2), order="F")
    im[1, 1, 0] = 99.0
    I, e, subs = problem.mask_images(im, 50.0)
    assert len(I) == 11
    assert list(e[:5]) == [1] * 5 and list(e[5:]) == [2] * 6
    assert 99.0 not in I


def test_psfconst_quirk():
    # equal rotations => "not constant" (imcom_proc.f90:593)
    assert problem.test_psfconst(["a", "a"], [0.0, 0.0]) == 0
    assert problem.test_psfconst(["a", "a"], [1.0, 2.0]) == 1
    assert problem.test_psfconst(["a", "b"], [1.0, 2.0]) == 0


def test_fortran_nint_and_npsf():
    assert problem.fortran_nint(2.5) == 3 and problem.fortran_nint(-2.5) == -3
    x = np.array([0.0, 11.7])
    assert problem.choose_npsf(x, x, x, x, 0.125, 0.125, (128, 128)) == 256
    assert problem.choose_npsf(x, x, x, x, 0.125, 0.125, (16, 16)) == 2 * 94


def test_build_Ndiag_blocks():
    assert list(problem.build_Ndiag(7, [1.0, 2.0])) == [1, 1, 1, 2, 2, 2, 2]


def test_synthetic_workloads_shapes():
    p = synth.make("small", 0)
    assert (p.n, p.m, p.nps, p.nexppsf, p.psfconst) == (576, 256, 256, 4, 0)
    assert np.all(np.diff(p.exp_i) >= 0)
    assert abs(p.G_unrot[:, :, 0].sum() - 1.0) < 1e-12
    q = synth.make_patch(3, 18)
    assert q.n < 4 * 18 * 18 and q.m == 24 * 24


def test_library_exports_every_header_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libimcom_gpu.so not built")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    syms = _lib.header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.SIGNATURES)


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.imcom_gpu_create(0, ctypes.byref(h)) != 0
    assert not h.value


def test_null_context_is_an_argument_error():
    """Argument checks come before any device work, so they hold without a GPU."""
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libimcom_gpu.so not built")
    lib = _lib.load()
    assert lib.imcom_gpu_build_image(None, None) == -1
    assert lib.imcom_gpu_build_images(None, 2, None, None) == -1
    assert lib.imcom_gpu_build_images_device(None, 2, None, 1, None, 1) == -1


def test_build_images_device_leading_dimensions():
    """The device entry gets each operand's row stride as its leading
    dimension; a single stack gets n and m whatever stride its length-1 axis
    carries."""
    import torch
    from imcom_b200.api import Solver
    s = Solver.__new__(Solver)
    s.n, s.m = 7, 5
    calls = []
    s._call = lambda name, *a: calls.append((name,) + a)
    one = torch.from_numpy(np.arange(7.0)[None, :])
    one = one.as_strided((1, 7), (1, 1))  # a length-1 axis with stride 1
    s.build_images_device(one, torch.zeros((1, 5), dtype=torch.float64))
    assert calls[-1][1] == 1 and calls[-1][3] == 7 and calls[-1][5] == 5
    wide_i = torch.zeros((3, 10), dtype=torch.float64)[:, :7]
    wide_h = torch.zeros((3, 9), dtype=torch.float64)[:, :5]
    s.build_images_device(wide_i, wide_h)
    assert calls[-1][1] == 3 and calls[-1][3] == 10 and calls[-1][5] == 9
    with pytest.raises(ValueError):
        s.build_images_device(torch.zeros((3, 8), dtype=torch.float64), wide_h)
