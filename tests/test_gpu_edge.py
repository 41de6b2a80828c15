"""Edge cases of the GPU solve path: masked (uneven) inputs, the constant-PSF
branch, iteration caps, state and argument errors."""
import numpy as np
import pytest

from imcom_b200 import EIGH_LIBRARY, EPS, ImcomError, synth
from oracle import oracle as O

from test_gpu_parity import EIG_MODE, rel

pytestmark = pytest.mark.gpu


@pytest.fixture()
def gs(solver):
    solver.set_eigensolver(EIG_MODE)
    return solver


def test_masked_patch_vs_oracle(gs):
    prob = synth.make_patch(seed=5, side=16, mask_frac=0.02)
    assert prob.n < 4 * 16 * 16 and prob.n % 32 != 0
    r_o = O.solve(prob, UnotS=True, US_max=1e-5, US_tol=1e-8, maxnits=53)
    r = gs.solve(prob, UnotS=True, US_max=1e-5, US_tol=1e-8, maxnits=53)
    assert rel(r.A, r_o.A) < 1e-12
    assert np.max(np.abs(r.L - r_o.L)) < 1e-12 * r_o.L.max()
    assert np.allclose(r.K, r_o.K, rtol=1e-6, atol=0)
    assert rel(r.T, r_o.T) < 1e-8
    assert np.allclose(r.S, r_o.S, rtol=1e-6)


def test_psfconst_branch(gs):
    prob = synth.make("tiny", 0)
    prob.G_unrot = np.asfortranarray(prob.G_unrot[:, :, :1])
    prob.rotangdeg = np.array([3.0, 7.0])  # one file, different angles: constant
    prob.psfconst = 1
    r_o = O.solve(prob, UnotS=True, US_max=1e-4, US_tol=1e-7, maxnits=40)
    r = gs.solve(prob, UnotS=True, US_max=1e-4, US_tol=1e-7, maxnits=40)
    assert rel(r.A, r_o.A) < 1e-12 and rel(r.B, r_o.B) < 1e-12
    assert rel(r.T, r_o.T) < 1e-8


def test_maxnits_zero_returns_kappa_min(gs):
    prob = synth.make("tiny", 0)
    r = gs.solve(prob, UnotS=True, US_max=1e-4, US_tol=1e-7, maxnits=0)
    assert np.allclose(r.K, r.kappa_min, rtol=1e-14)
    assert np.all(r.nevals == 1)


def test_state_and_argument_errors(solver):
    prob = synth.make("tiny", 0)
    solver.set_problem(prob)
    solver.load_K(np.ones(prob.m))
    with pytest.raises(ImcomError) as e:
        solver.build_image()  # T not built yet
    assert e.value.status == 3
    with pytest.raises(ImcomError) as e:
        solver.set_psfs(prob.G_unrot, prob.rotangdeg, prob.Gamma, psfconst=2)
    assert e.value.status == -4
    bad = prob.x_i.copy()
    bad[3] = np.nan
    with pytest.raises(ImcomError) as e:
        solver.set_inputs(bad, prob.y_i, prob.exp_i, prob.X_a, prob.Y_a)
    assert e.value.status == 7
    with pytest.raises(ImcomError):
        solver.set_inputs(prob.x_i, prob.y_i, prob.exp_i[::-1], prob.X_a, prob.Y_a)


def test_nonfinite_psf_is_rejected(solver):
    """A NaN or inf in the PSF arrays is reported with its index (checked on
    the device after the upload) and leaves no usable PSF state behind."""
    prob = synth.make("tiny", 0)
    solver.set_problem(prob)
    G = np.array(prob.G_unrot, order="F")
    G.ravel(order="F")[1234] = np.nan
    with pytest.raises(ImcomError) as ex:
        solver.set_psfs(G, prob.rotangdeg, prob.Gamma, prob.psfconst)
    assert ex.value.status == 7 and "G_unrot" in str(ex.value) and "1234" in str(ex.value)
    with pytest.raises(ImcomError):
        solver.psf_spectra()
    Gam = np.array(prob.Gamma, order="F")
    Gam[3, 5] = np.inf
    with pytest.raises(ImcomError) as ex:
        solver.set_psfs(prob.G_unrot, prob.rotangdeg, Gam, prob.psfconst)
    assert ex.value.status == 7 and "Gamma" in str(ex.value)
    solver.set_problem(prob)  # a clean upload works again
    assert solver.psf_spectra() > 0


def test_cached_system_path_reuses_T(gs):
    """T-reuse path (imcom_bisect.f90:47-62): H from a loaded T equals H of the solve."""
    prob = synth.make("tiny", 0)
    r = gs.solve(prob, UnotS=True, US_max=1e-4, US_tol=1e-7, maxnits=40)
    gs.load_T(r.T)
    H = gs.build_image()
    assert rel(H, r.H) < 1e-14
