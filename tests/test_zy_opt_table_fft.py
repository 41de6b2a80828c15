"""The lookup tables through the library's own pruned, fused inverse FFT
(IMCOM_OPT_TABLE_FFT = 1, imcom_b200/csrc/table_fft.cu), through the C-ABI:
A and B against the golden fixtures and the oracle at the cuFFT path's bars
(1e-12 of the largest entry), on table sides that use every radix of the
transform (L = 288: 4 4 2 3 3; 270: 2 3 3 3 5; 420: 4 3 5 7; 330: 2 3 5 11;
390: 2 3 5 13; 768: 4 4 4 4 3), and a side with a prime factor above 13
(L = 306 = 2 3 3 17), which stays on cuFFT and so matches the default path bit
for bit.  Each test runs its own
context so the option does not reach other tests."""
import os
import sys

import numpy as np
import pytest

from imcom_b200 import Solver, synth
from imcom_b200.api import OPT_TABLE_FFT, TABLE_FFT_CUFFT, TABLE_FFT_OWN
from oracle import oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def build_AB(prob, mode):
    with Solver(0) as s:
        s.set_option(OPT_TABLE_FFT, mode)
        s.set_problem(prob)
        s.psf_spectra()
        return s.build_A(), s.build_B()


@pytest.mark.parametrize("case", ["tiny_u", "tiny_rot"])
def test_own_table_fft_golden(case):
    prob, d = make_golden.load(case)
    A, B = build_AB(prob, TABLE_FFT_OWN)
    assert np.array_equal(A, A.T)
    assert rel(A, d["A"]) < 1e-12
    assert rel(B, d["B"]) < 1e-12


@pytest.mark.parametrize("workload,stamp,side", [("tiny", 48, 288), ("tiny", 40, 270),
                                                 ("tiny", 70, 420), ("tiny", 55, 330),
                                                 ("tiny", 65, 390), ("small", 128, 768)])
def test_own_table_fft_vs_oracle(workload, stamp, side):
    prob = synth.make(workload, 0, psf_stamp=stamp)
    assert 3 * prob.nps == side
    r = O.solve(prob, UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=40)
    A, B = build_AB(prob, TABLE_FFT_OWN)
    assert rel(A, r.A) < 1e-12
    assert rel(B, r.B) < 1e-12


def test_side_with_large_prime_stays_on_cufft():
    prob = synth.make("tiny", 0, psf_stamp=51)
    assert 3 * prob.nps == 306
    A1, B1 = build_AB(prob, TABLE_FFT_OWN)
    A0, B0 = build_AB(prob, TABLE_FFT_CUFFT)
    assert np.array_equal(A1, A0) and np.array_equal(B1, B0)


def test_register_path_matches_cufft_at_nps_576():
    """nps = 576, L = 1728 (the n = 4096 workload's sides) takes the register
    path: three length-576 transforms of pre-twiddled copies per line, one
    warp per line.  A and B against the cuFFT path at the same bar."""
    prob = synth.make("n4096", 0)
    assert prob.nps == 576
    A1, B1 = build_AB(prob, TABLE_FFT_OWN)
    A0, B0 = build_AB(prob, TABLE_FFT_CUFFT)
    assert np.array_equal(A1, A1.T)
    assert rel(A1, A0) < 1e-12
    assert rel(B1, B0) < 1e-12
