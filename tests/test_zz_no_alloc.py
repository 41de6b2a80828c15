"""imcom_gpu_build_P_noalloc: the allocation-free projection P = Q^T B.

Callers that cannot allocate device memory (their GPU memory is reserved up
front by their own allocator) pass device buffers they already own; the entry
point keeps its split-K partial sums in a fixed device array instead of
allocating.  This file runs last so a failure here leaves every other test
already run.  The check: two calls in a row through the C-ABI agree with
imcom_gpu_build_P's P (normwise relative difference < 1e-13, the tolerance of
the other P tests).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

IMCOM_ERR_NOALLOC_SIZE = 8


def test_build_P_noalloc_matches_build_P(solver):
    import torch

    from imcom_b200 import EIGH_DC, synth

    prob = synth.make("small", seed=3)
    solver.set_eigensolver(EIGH_DC)
    r = solver.solve(prob, UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=40)
    n, m = prob.n, prob.m
    # the caller's own device buffers (column-major, ld = n)
    dQ = torch.tensor(np.asfortranarray(r.Q).ravel(order="F"), device="cuda")
    dB = torch.tensor(np.asfortranarray(r.B).ravel(order="F"), device="cuda")
    lib = solver.lib
    scale = np.abs(r.P).max()
    for call in range(2):
        dP = torch.full((n * m,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        st = lib.imcom_gpu_build_P_noalloc(dQ.data_ptr(), n, dB.data_ptr(), n, dP.data_ptr(), n,
                                           n, m, None)
        assert st == 0, f"call {call}: status {st}"
        torch.cuda.synchronize()
        P = dP.cpu().numpy().reshape((n, m), order="F")
        assert np.max(np.abs(P - r.P)) < 1e-13 * scale, f"call {call}"


def test_build_P_noalloc_odd_leading_dimensions_on_a_stream(solver):
    """Operands that are views with odd leading dimensions (the kernel's 8-byte
    copy path) and the caller's own CUDA stream: the same P, twice."""
    import torch

    from imcom_b200 import EIGH_DC, synth

    prob = synth.make("small", seed=4)
    solver.set_eigensolver(EIGH_DC)
    r = solver.solve(prob, UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=40)
    n, m = prob.n, prob.m
    ld = n + 1  # odd: columns start on 8-byte boundaries only

    def padded(M):
        buf = np.zeros((ld, M.shape[1]), order="F")
        buf[:n, :] = M
        return torch.tensor(buf.ravel(order="F"), device="cuda")

    dQ, dB = padded(r.Q), padded(r.B)
    lib = solver.lib
    scale = np.abs(r.P).max()
    stream = torch.cuda.Stream()
    for call in range(2):
        dP = torch.full((ld * m,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        st = lib.imcom_gpu_build_P_noalloc(dQ.data_ptr(), ld, dB.data_ptr(), ld, dP.data_ptr(), ld,
                                           n, m, ctypes.c_void_p(stream.cuda_stream))
        assert st == 0, f"call {call}: status {st}"
        stream.synchronize()
        P = dP.cpu().numpy().reshape((ld, m), order="F")[:n]
        assert np.max(np.abs(P - r.P)) < 1e-13 * scale, f"call {call}"


def test_build_P_noalloc_rejects_oversized_problem(solver):
    lib = solver.lib
    n = m = 4096  # 2 * 4096 * 4096 partial sums exceed the fixed array
    fake = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    st = lib.imcom_gpu_build_P_noalloc(fake, n, fake, n, fake, n, n, m, None)
    assert st == IMCOM_ERR_NOALLOC_SIZE
    assert lib.imcom_gpu_build_P_noalloc(None, n, fake, n, fake, n, n, m, None) == -1
    # small n, but more output columns than one launch grid can index
    n, m = 32, 65536
    st = lib.imcom_gpu_build_P_noalloc(fake, n, fake, n, fake, n, n, m, None)
    assert st == IMCOM_ERR_NOALLOC_SIZE
