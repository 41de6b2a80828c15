"""In-memory IMCOM problem: the module state the reference driver assembles
before the solve path starts (imcom_data.f90:24-135).

The helpers here restate the host-side set-up the reference keeps in Fortran
(imcom_io / imcom_proc) so that synthetic inputs reach the solve path in
exactly the layout the reference would hand to it:

* ``mask_images``     imcom_alloc_gims (imcom_io.f90:36-129): mask = I < saturation,
                      exposure-major flattening, 1-based ``exp_i``.
* ``grid_xy``         imcom_build_xy (imcom_proc.f90:56-89) / imcom_xarr / imcom_yarr.
* ``grid_XaYa``       imcom_build_XaYa (imcom_proc.f90:93-119).
* ``pad_psfs``        imcom_alloc_psfs (imcom_io.f90:244-335): n1psf choice, centred
                      zero-padding and normalisation to unit sum.
* ``test_psfconst``   imcom_test_psfconst (imcom_proc.f90:582-599), including its
                      equal-rotation quirk.
* ``build_Ndiag``     imcom_build_Ndiag (imcom_matrix.f90:556-582).

Arrays use Fortran (column-major) order: an image is indexed (x, y) with x
fastest.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Problem:
    """Inputs of the solve path (everything imcom.f90 has set up by line 122)."""

    x_i: np.ndarray          # (n,) input pixel x, input-pixel units
    y_i: np.ndarray          # (n,)
    exp_i: np.ndarray        # (n,) int32, 1-based exposure index
    I_i: np.ndarray          # (n,) unmasked pixel values
    X_a: np.ndarray          # (m,) output pixel x (x fastest over the n1out x n2out grid)
    Y_a: np.ndarray          # (m,)
    n1out: int
    n2out: int
    G_unrot: np.ndarray      # (nps, nps, nexppsf) padded, unit-sum PSFs
    Gamma: np.ndarray        # (nps, nps) padded, unit-sum target PSF
    rotangdeg: np.ndarray    # (nexp,) PSF rotation angles, degrees
    noise: np.ndarray        # (nexp,) per-exposure noise
    psfxscale: float
    psfyscale: float
    psfconst: int
    name: str = "problem"
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.x_i.shape[0])

    @property
    def m(self) -> int:
        return int(self.X_a.shape[0])

    @property
    def nps(self) -> int:
        return int(self.G_unrot.shape[0])

    @property
    def nexp(self) -> int:
        return int(self.noise.shape[0])

    @property
    def nexppsf(self) -> int:
        return int(self.G_unrot.shape[2])


def xarr(n1: int, n2: int) -> np.ndarray:
    """imcom_xarr: x = (i - 1) along the first axis."""
    return np.asfortranarray(np.repeat(np.arange(n1, dtype=np.float64)[:, None], n2, axis=1))


def yarr(n1: int, n2: int) -> np.ndarray:
    """imcom_yarr = transpose(imcom_xarr(n2, n1))."""
    return np.asfortranarray(xarr(n2, n1).T)


def mask_images(images: np.ndarray, saturation: float):
    """imcom_alloc_gims: images (n1gim, n2gim, nexp) -> (I_i, exp_i, mask_subs_i).

    ``mask_subs_i`` is 0-based here.  Pixels with I >= saturation (and NaN)
    are dropped.
    """
    n1, n2, nexp = images.shape
    I_unmasked = images.reshape(-1, order="F")
    exp_unmasked = np.repeat(np.arange(1, nexp + 1, dtype=np.int32), n1 * n2)
    mask = I_unmasked < saturation
    subs = np.nonzero(mask)[0]
    return I_unmasked[subs].copy(), exp_unmasked[subs].copy(), subs


def grid_xy(n1gim, n2gim, gimxscale, gimyscale, dither):
    """imcom_build_xy before masking: x_unmasked (n1gim, n2gim, nexp)."""
    nexp = len(gimxscale)
    xu = np.zeros((n1gim, n2gim, nexp), order="F")
    yu = np.zeros((n1gim, n2gim, nexp), order="F")
    for i in range(nexp):
        xu[:, :, i] = xarr(n1gim, n2gim) * gimxscale[i] + dither[i][0]
        yu[:, :, i] = yarr(n1gim, n2gim) * gimyscale[i] + dither[i][1]
    return xu, yu


def grid_XaYa(n1out, n2out, outxscale, outyscale, outpos1, outpos2):
    """imcom_build_XaYa: X_a, Y_a flattened column-major (x fastest)."""
    Xa = xarr(n1out, n2out) * outxscale + outpos1
    Ya = yarr(n1out, n2out) * outyscale + outpos2
    return Xa.reshape(-1, order="F").copy(), Ya.reshape(-1, order="F").copy()


def fortran_nint(v: float) -> int:
    """Fortran NINT: round half away from zero."""
    return int(np.sign(v) * np.floor(abs(v) + 0.5))


def choose_npsf(x_i, y_i, X_a, Y_a, psfxscale, psfyscale, psf_shape) -> int:
    """imcom_alloc_psfs (imcom_io.f90:279-286): the padded PSF side n1psf."""
    n1pad = 2 * fortran_nint((max(x_i.max(), X_a.max()) - min(x_i.min(), X_a.min())) / psfxscale)
    n2pad = 2 * fortran_nint((max(y_i.max(), Y_a.max()) - min(y_i.min(), Y_a.min())) / psfyscale)
    n1pad = max(n1pad, n2pad)
    n2pad = n1pad
    if n1pad < psf_shape[0] * 2 or n2pad < psf_shape[1] * 2:
        n1pad = max(psf_shape[0] * 2, psf_shape[1] * 2)
    return int(n1pad)


def pad_psf(stamp: np.ndarray, nps: int) -> np.ndarray:
    """Centre a PSF stamp in an (nps, nps) zero array and normalise to unit sum
    (imcom_io.f90:306-329)."""
    p1, p2 = stamp.shape
    out = np.zeros((nps, nps), order="F")
    n1min = (nps - p1) // 2
    n2min = (nps - p2) // 2
    out[n1min:n1min + p1, n2min:n2min + p2] = stamp / stamp.sum()
    return out


def test_psfconst(psffiles, rotangdeg) -> int:
    """imcom_test_psfconst (imcom_proc.f90:582-599).

    Mirrors the reference exactly: the PSF counts as *not* constant when a
    file name differs OR when a rotation angle EQUALS the first one.
    """
    for i in range(1, len(psffiles)):
        if psffiles[i] != psffiles[0] or abs(rotangdeg[i] - rotangdeg[0]) <= 1e-15:
            return 0
    return 1


def build_Ndiag(n: int, noise) -> np.ndarray:
    """imcom_build_Ndiag: noise(e) over contiguous blocks of n/nexp."""
    nexp = len(noise)
    out = np.zeros(n)
    for i in range(1, nexp + 1):
        n_i = 1 + (i - 1) * (n // nexp)
        n_f = i * (n // nexp) if i != nexp else n
        out[n_i - 1:n_f] = noise[i - 1]
    return out
