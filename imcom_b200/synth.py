"""Seeded synthetic IMCOM inputs.

The reference measures nothing on a public dataset; its paper tests
(tests/paper_test/make_testimages6v2_rt5.pro, testimage2v0.pro,
pix_response2v0.pro, charge_diff2v0.pro) build dithered exposures of an
exponential-profile sky seen through a PSF convolved with a top-hat pixel
response.  This module follows that recipe with numpy so every workload can be
regenerated from a seed:

* ``gaussian_pixel_psf``  Gaussian PSF convolved with the top-hat pixel (OTF =
  Gaussian x sinc x sinc), sampled at ``psfscale`` input pixels.
* ``airy_pixel_psf``      obscured-aperture PSF |FT(pupil)|^2 with the given
  lambda/D (input pixels), convolved with the pixel.
* ``gaussian_psf``        target PSF Gamma.

Workloads (``make``):

* ``small``   4 x 12x12 exposures (n=576), uniform [0,1) dithers, no rotation,
              Gaussian sigma=0.6 px (x) pixel PSF in a 128^2 stamp at 1/8 px
              (nps=256, lookup side 768), Gamma Gaussian sigma=0.8 px, 16x16
              output at 0.5 px over the central region.
* ``n4096``   4 x 32x32 exposures (n=4096), rotations U[-5,5] deg, uniform
              dithers, Airy lambda/D=0.5 px (x) pixel in a 288^2 stamp
              (nps=576, lookup side 1728), Gamma sigma=0.9 px, 64x64 output at
              0.5 px (m=4096).
* ``n16200``  8 x 45x45 exposures (n=16200), rotations U[-10,10] deg, Airy
              lambda/D=0.6 px, Gamma sigma=1.0 px, 128x128 output (m=16384).
* ``tiny``    2 x 6x6 exposures, for fast unit tests.

Each exposure names its own PSF file so the per-exposure table path is taken
(imcom_test_psfconst would otherwise apply only the first rotation).
"""
from __future__ import annotations

import numpy as np

from .problem import (Problem, build_Ndiag, choose_npsf, grid_XaYa, grid_xy, mask_images,
                      pad_psf, test_psfconst)


def _freqs(P: int, psfscale: float):
    k = np.fft.fftfreq(P, d=psfscale)  # cycles per input pixel
    return np.meshgrid(k, k, indexing="ij")


def _from_otf(otf: np.ndarray) -> np.ndarray:
    img = np.fft.fftshift(np.real(np.fft.ifft2(otf)))
    return np.asfortranarray(img)


def gaussian_psf(P: int, psfscale: float, sigma: float) -> np.ndarray:
    kx, ky = _freqs(P, psfscale)
    return _from_otf(np.exp(-2.0 * np.pi ** 2 * sigma ** 2 * (kx ** 2 + ky ** 2)))


def gaussian_pixel_psf(P: int, psfscale: float, sigma: float) -> np.ndarray:
    kx, ky = _freqs(P, psfscale)
    otf = np.exp(-2.0 * np.pi ** 2 * sigma ** 2 * (kx ** 2 + ky ** 2)) * np.sinc(kx) * np.sinc(ky)
    return _from_otf(otf)


def airy_pixel_psf(P: int, psfscale: float, lam_over_d: float, obscuration: float = 0.3) -> np.ndarray:
    kx, ky = _freqs(P, psfscale)
    kr = np.hypot(kx, ky)
    rpupil = 0.5 / lam_over_d  # pupil radius in cycles/px: OTF cutoff D/lambda
    pupil = ((kr <= rpupil) & (kr >= obscuration * rpupil)).astype(np.float64)
    amp = np.fft.ifft2(pupil)
    psf = np.abs(amp) ** 2
    otf = np.fft.fft2(psf) * np.sinc(kx) * np.sinc(ky)
    return _from_otf(otf)


def _sky(x, y, rng, nobj, extent, cx, cy):
    """Exponential-profile galaxies (testimage2v0.pro:1-6 shape) at positions."""
    v = np.zeros_like(x)
    for _ in range(nobj):
        x0 = cx + (rng.random() - 0.5) * extent
        y0 = cy + (rng.random() - 0.5) * extent
        r0 = 0.5 + 1.5 * rng.random()
        amp = 20.0 + 80.0 * rng.random()
        q = 0.5 + 0.5 * rng.random()
        th = np.pi * rng.random()
        dx, dy = x - x0, y - y0
        u = dx * np.cos(th) + dy * np.sin(th)
        w = (-dx * np.sin(th) + dy * np.cos(th)) / q
        v += amp * np.exp(-np.hypot(u, w) / r0)
    return v


def build_problem(*, name, nexp, side, rot_range, psf_kind, psf_param, psf_stamp, gamma_sigma,
                  n_out, out_scale, seed, psfscale=0.125, noise=1.0, mask_frac=0.0,
                  saturation=None) -> Problem:
    rng = np.random.default_rng(seed)
    dithers = [(rng.random(), rng.random()) for _ in range(nexp)]
    rots = ([(rng.random() * 2.0 - 1.0) * rot_range for _ in range(nexp)]
            if rot_range > 0 else [0.0] * nexp)
    # Input positions (imcom_build_xy, or user x/y maps when rotated).
    xu, yu = grid_xy(side, side, [1.0] * nexp, [1.0] * nexp, [(0.0, 0.0)] * nexp)
    c = (side - 1) / 2.0
    for e in range(nexp):
        th = np.deg2rad(rots[e])
        px, py = xu[:, :, e] - c, yu[:, :, e] - c
        xu[:, :, e] = c + np.cos(th) * px - np.sin(th) * py + dithers[e][0]
        yu[:, :, e] = c + np.sin(th) * px + np.cos(th) * py + dithers[e][1]
    # Sky values with unit Gaussian noise (NOISE 1.0).
    images = np.zeros((side, side, nexp), order="F")
    sky_rng = np.random.default_rng(seed + 1000)
    nobj = max(2, side // 4)
    state = sky_rng.bit_generator.state
    for e in range(nexp):
        sky_rng.bit_generator.state = state
        images[:, :, e] = _sky(xu[:, :, e], yu[:, :, e], sky_rng, nobj, side * 0.8, c, c)
    images += noise * rng.standard_normal(images.shape)
    if mask_frac > 0.0:
        sat = 1e30 if saturation is None else saturation
        bad = rng.random(images.shape) < mask_frac
        images[bad] = sat
        saturation = sat
    if saturation is None:
        saturation = np.finfo(np.float64).max  # DLAMCH('O'), the CLI default
    I_i, exp_i, subs = mask_images(images, saturation)
    x_i = xu.reshape(-1, order="F")[subs].copy()
    y_i = yu.reshape(-1, order="F")[subs].copy()
    # Output grid over the central region.
    span = (n_out - 1) * out_scale
    outpos = c + 0.5 - span / 2.0
    X_a, Y_a = grid_XaYa(n_out, n_out, out_scale, out_scale, outpos, outpos)
    psffiles = [f"psf{e + 1}.fits" for e in range(nexp)]
    psfconst = test_psfconst(psffiles, rots)
    nexppsf = 1 if psfconst else nexp
    nps = choose_npsf(x_i, y_i, X_a, Y_a, psfscale, psfscale, (psf_stamp, psf_stamp))
    G = np.zeros((nps, nps, nexppsf), order="F")
    for e in range(nexppsf):
        if psf_kind == "gaussian":
            stamp = gaussian_pixel_psf(psf_stamp, psfscale, psf_param[e] if np.ndim(psf_param) else psf_param)
        else:
            stamp = airy_pixel_psf(psf_stamp, psfscale, psf_param)
        G[:, :, e] = pad_psf(stamp, nps)
    Gamma = pad_psf(gaussian_psf(psf_stamp, psfscale, gamma_sigma), nps)
    return Problem(x_i=x_i, y_i=y_i, exp_i=exp_i.astype(np.int32), I_i=I_i, X_a=X_a, Y_a=Y_a,
                   n1out=n_out, n2out=n_out, G_unrot=G, Gamma=Gamma,
                   rotangdeg=np.array(rots, dtype=np.float64),
                   noise=np.full(nexp, noise, dtype=np.float64), psfxscale=psfscale,
                   psfyscale=psfscale, psfconst=psfconst, name=name,
                   meta=dict(seed=seed, dithers=dithers, psfstamp=psf_stamp,
                             saturation=float(saturation)))


WORKLOADS = {
    "tiny": dict(nexp=2, side=6, rot_range=0.0, psf_kind="gaussian", psf_param=0.6,
                 psf_stamp=48, gamma_sigma=0.8, n_out=6, out_scale=0.5),
    "small": dict(nexp=4, side=12, rot_range=0.0, psf_kind="gaussian", psf_param=0.6,
                  psf_stamp=128, gamma_sigma=0.8, n_out=16, out_scale=0.5),
    "small_rot": dict(nexp=4, side=12, rot_range=5.0, psf_kind="airy", psf_param=0.5,
                      psf_stamp=128, gamma_sigma=0.9, n_out=16, out_scale=0.5),
    "n4096": dict(nexp=4, side=32, rot_range=5.0, psf_kind="airy", psf_param=0.5,
                  psf_stamp=288, gamma_sigma=0.9, n_out=64, out_scale=0.5),
    "n16200": dict(nexp=8, side=45, rot_range=10.0, psf_kind="airy", psf_param=0.6,
                   psf_stamp=432, gamma_sigma=1.0, n_out=128, out_scale=0.5),
}


def make(workload: str, seed: int = 0, **over) -> Problem:
    kw = dict(WORKLOADS[workload])
    kw.update(over)
    return build_problem(name=workload, seed=seed, **kw)


def make_patch(seed: int, side: int, mask_frac: float = 0.02) -> Problem:
    """One patch of the batched-patch workload: 4 exposures of ``side``^2 px,
    ``mask_frac`` of pixels masked, Gaussian PSF sigma ~ U[0.5, 0.8] per
    exposure, 24x24 output at 0.5 px."""
    rng = np.random.default_rng(10_000 + seed)
    sig = 0.5 + 0.3 * rng.random(4)
    return build_problem(name=f"patch{seed}", nexp=4, side=side, rot_range=0.0,
                         psf_kind="gaussian", psf_param=sig, psf_stamp=64, gamma_sigma=0.8,
                         n_out=24, out_scale=0.5, seed=seed, mask_frac=mask_frac)


__all__ = ["make", "make_patch", "build_problem", "WORKLOADS", "gaussian_psf",
           "gaussian_pixel_psf", "airy_pixel_psf", "build_Ndiag"]
