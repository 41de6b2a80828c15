"""T applied to many image stacks: imcom_gpu_build_images(_device) against
the per-stack H_a = sum_i T_ia I_i of imcom_build_image
(imcom_matrix.f90:754-790), through the C-ABI.

FP64 sums in any order differ from the exact H by at most
n * eps * (|T|^T |I|) (the standard bound for an n-term dot product); the
tests hold each element to twice that.
"""
import numpy as np
import pytest

from imcom_b200.api import EPS, Solver
from imcom_b200._lib import ImcomError

pytestmark = pytest.mark.gpu

IMCOM_ERR_STATE = 3


def geometry(s, n, m, seed):
    rng = np.random.default_rng(seed)
    s.set_inputs(rng.uniform(0, 30, n), rng.uniform(0, 30, n), np.ones(n, dtype=np.int32),
                 rng.uniform(0, 30, m), rng.uniform(0, 30, m), I_i=rng.standard_normal(n))
    return rng


def check(H, T, I):
    n = T.shape[0]
    ref = T.T @ I
    bound = 2.0 * n * EPS * (np.abs(T).T @ np.abs(I))
    assert H.shape == ref.shape
    assert np.all(np.abs(H - ref) <= bound + 1e-300)


@pytest.mark.parametrize("n,m,stacks", [(300, 500, 1), (300, 500, 3), (300, 500, 129),
                                        (1031, 257, 64)])
def test_build_images_matches_per_stack_sums(n, m, stacks):
    with Solver(0) as s:
        rng = geometry(s, n, m, n + stacks)
        T = np.asfortranarray(rng.standard_normal((n, m)) * np.exp(rng.uniform(-3, 3, (n, 1))))
        I = np.asfortranarray(rng.standard_normal((n, stacks)) + 5.0)
        s.load_T(T)
        check(s.build_images(I), T, I)
        # the first stack through the one-stack path agrees within the same bound
        s.set_inputs(*s._keep[:2], s._keep[6], *s._keep[2:4], I_i=I[:, 0])
        s.load_T(T)
        check(s.build_image()[:, None], T, I[:, :1])


def test_build_images_device_strided():
    torch = pytest.importorskip("torch")
    n, m, stacks = 301, 203, 17
    with Solver(0) as s:
        rng = geometry(s, n, m, 7)
        T = np.asfortranarray(rng.standard_normal((n, m)))
        s.load_T(T)
        I = rng.standard_normal((n, stacks))
        # rows of wider tensors: leading dimensions n + 4 = 305 (odd, so the
        # GEMM takes its 8-byte operand path) and m + 3
        dIw = torch.zeros((stacks, n + 4), dtype=torch.float64, device="cuda")
        dIw[:, :n] = torch.from_numpy(I.T.copy()).cuda()
        dHw = torch.full((stacks, m + 3), 7.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        s.build_images_device(dIw[:, :n], dHw[:, :m])
        s.synchronize()
        Hw = dHw.cpu().numpy()
        check(Hw[:, :m].T, T, I)
        assert np.all(Hw[:, m:] == 7.0)  # nothing written past m
        # one stack, whatever stride its length-1 axis carries
        d1 = torch.from_numpy(np.ascontiguousarray(I[:, :1].T)).to("cuda")
        h1 = torch.empty((1, m), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        s.build_images_device(d1, h1)
        s.synchronize()
        check(h1.cpu().numpy().T, T, I[:, :1])


def test_build_images_errors():
    with Solver(0) as s:
        geometry(s, 40, 30, 1)
        with pytest.raises(ImcomError) as e:
            s.build_images(np.zeros((40, 2)))
        assert e.value.status == IMCOM_ERR_STATE
        s.load_T(np.zeros((40, 30), order="F"))
        assert s.build_images(np.zeros((40, 0))).shape == (30, 0)
        with pytest.raises(ValueError):
            s.build_images(np.zeros((41, 2)))
        assert s.lib.imcom_gpu_build_images(s.h, -1, None, None) == -2
        assert s.lib.imcom_gpu_build_images_device(s.h, 0, None, 39, None, 30) == -4
        assert s.lib.imcom_gpu_build_images_device(s.h, 0, None, 40, None, 29) == -6
