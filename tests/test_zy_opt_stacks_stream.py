"""The streaming kernel of imcom_gpu_build_images (IMCOM_OPT_STACK_KERNEL = 1,
stacks_kernel in imcom_b200/csrc/solve.cu) through the C-ABI: H = T^T I
within twice the n-term dot-product bound n * eps * (|T|^T |I|), for one,
two, three and eight stacks (one pass of 1, 2, 4 and 8), and for 9 and 19
stacks (two and three passes, the last one short), with m not a multiple of
the 16 columns a block holds and n not a multiple of the 128-row chunk; and
on strided device operands (odd leading dimensions).  Each test runs its own
context so the option does not reach other tests."""
import numpy as np
import pytest

from imcom_b200.api import EPS, OPT_STACK_KERNEL, STACKS_STREAM, Solver

pytestmark = pytest.mark.gpu


def check(H, T, I):
    n = T.shape[0]
    bound = 2.0 * n * EPS * (np.abs(T).T @ np.abs(I))
    assert H.shape == (T.shape[1], I.shape[1])
    assert np.all(np.abs(H - T.T @ I) <= bound + 1e-300)


def stream_solver(n, m, seed):
    s = Solver(0)
    s.set_option(OPT_STACK_KERNEL, STACKS_STREAM)
    rng = np.random.default_rng(seed)
    s.set_inputs(rng.uniform(0, 30, n), rng.uniform(0, 30, n), np.ones(n, dtype=np.int32),
                 rng.uniform(0, 30, m), rng.uniform(0, 30, m))
    return s, rng


@pytest.mark.parametrize("stacks", [1, 2, 3, 8, 9, 19])
def test_stream_kernel_matches_dot_products(stacks):
    n, m = 301, 203
    s, rng = stream_solver(n, m, stacks)
    with s:
        T = np.asfortranarray(rng.standard_normal((n, m)) * np.exp(rng.uniform(-3, 3, (n, 1))))
        I = np.asfortranarray(rng.standard_normal((n, stacks)) + 5.0)
        s.load_T(T)
        check(s.build_images(I), T, I)


def test_stream_kernel_strided_device_operands():
    torch = pytest.importorskip("torch")
    n, m, stacks = 257, 131, 11
    s, rng = stream_solver(n, m, 7)
    with s:
        T = np.asfortranarray(rng.standard_normal((n, m)))
        s.load_T(T)
        I = rng.standard_normal((n, stacks))
        dIw = torch.zeros((stacks, n + 2), dtype=torch.float64, device="cuda")  # ld 259
        dIw[:, :n] = torch.from_numpy(I.T.copy()).cuda()
        dHw = torch.full((stacks, m + 4), 7.0, dtype=torch.float64, device="cuda")  # ld 135
        torch.cuda.synchronize()
        s.build_images_device(dIw[:, :n], dHw[:, :m])
        s.synchronize()
        Hw = dHw.cpu().numpy()
        check(Hw[:, :m].T, T, I)
        assert np.all(Hw[:, m:] == 7.0)  # nothing written past m
