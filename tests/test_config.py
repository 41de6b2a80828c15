"""Configuration reader (imcom_b200.config) on the reference's own example
(example/userxy1, fixture tests/golden/example_userxy1.npz) and on written
USERXY = 0 configurations: the inputs it assembles are the ones the
reference's driver builds (imcom_io.f90:499-971, imcom.f90:56-84)."""
import os
import sys

import numpy as np
import pytest

from imcom_b200 import config, fits, problem

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_example_fixture  # noqa: E402


@pytest.fixture(scope="module")
def example_dir(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("userxy1"))
    return make_example_fixture.unpack(d)


def test_example_config_fields(example_dir):
    cfg = config.read_config(example_dir)
    assert (cfg.psfxscale, cfg.psfyscale, cfg.nexp, cfg.userxy) == (0.1, 0.1, 4, 1)
    assert cfg.psffile == ["psf.example.fits"] * 4
    assert cfg.gimfile == [f"test{i}.example.fits" for i in range(1, 5)]
    assert cfg.gimxfile == [f"x{i}.example.fits" for i in range(1, 5)]
    assert cfg.rotangdeg == [0.0] * 4 and cfg.noise == [1.0] * 4
    assert cfg.gamfile == "psf.example.fits"
    assert cfg.outfiles["H"] == "H.example.fits" and cfg.outfiles["U"] == "U.example.fits"
    assert (cfg.outxfile, cfg.outyfile) == ("xout.example.fits", "yout.example.fits")
    assert cfg.cachefiles == {k: f"{k}.example.fits" for k in "ABQLP"}


def test_example_problem_matches_the_files(example_dir):
    d = os.path.dirname(example_dir)
    prob = config.load_problem(example_dir)
    assert (prob.n, prob.m, prob.nps, prob.nexppsf, prob.psfconst) == (4096, 4225, 640, 4, 0)
    # exposure-major flattening (imcom_alloc_gims), x fastest within an exposure
    im2 = fits.read(os.path.join(d, "test2.example.fits"))
    assert np.array_equal(prob.I_i[1024:2048], im2.reshape(-1, order="F"))
    assert np.array_equal(prob.exp_i, np.repeat(np.arange(1, 5, dtype=np.int32), 1024))
    x3 = fits.read(os.path.join(d, "x3.example.fits"))
    assert np.array_equal(prob.x_i[2048:3072], x3.reshape(-1, order="F"))
    Xa = fits.read(os.path.join(d, "xout.example.fits"))
    assert np.array_equal(prob.X_a, Xa.reshape(-1, order="F"))
    # PSFs centred in the padded array at unit sum (imcom_alloc_psfs)
    assert prob.G_unrot.shape == (640, 640, 4)
    assert np.allclose(prob.G_unrot.sum(axis=(0, 1)), 1.0, rtol=1e-14)
    psf = fits.read(os.path.join(d, "psf.example.fits"))
    assert np.allclose(prob.Gamma[192:448, 192:448], psf / psf.sum(), rtol=0, atol=1e-18)
    assert prob.Gamma[:192].sum() == 0.0


def test_saturation_masks_pixels(example_dir):
    prob = config.load_problem(example_dir, saturation=20.0)
    full = config.load_problem(example_dir)
    keep = full.I_i < 20.0
    assert prob.n == int(keep.sum()) < full.n
    assert np.array_equal(prob.I_i, full.I_i[keep])
    assert np.array_equal(prob.x_i, full.x_i[keep])
    assert np.array_equal(prob.exp_i, full.exp_i[keep])


def test_userxy0_grid_configuration(tmp_path):
    """USERXY = 0: coordinates built from scales and dithers
    (imcom_build_xy / imcom_build_XaYa)."""
    rng = np.random.default_rng(3)
    for i in range(1, 3):
        fits.write(str(tmp_path / f"im{i}.fits"), rng.random((6, 5)))
    stamp = np.exp(-((np.arange(16) - 7.5) ** 2)[:, None] / 4 - ((np.arange(16) - 7.5) ** 2)[None] / 4)
    fits.write(str(tmp_path / "psf.fits"), stamp)
    for i, (rot, dx, dy) in enumerate([(0.0, 0.0, 0.0), (3.0, 0.25, -0.5)], start=1):
        (tmp_path / f"in{i}").write_text(
            "PSFFILE     psf.fits\n"
            f"GIMFILE     im{i}.fits\n"
            f"ROTANGDEG   {rot}\n"
            "NOISE       2.0d0\n"
            "GIMXSCALE   1.0\n"
            "GIMYSCALE   1.0\n"
            f"DITHER      {dx} {dy}\n")
    (tmp_path / "out").write_text(
        "GAMFILE     psf.fits\nOUTFILE     H.fits\nKFILE       K.fits\nTFILE       T.fits\n"
        "SFILE       S.fits\nUFILE       U.fits\nOUTXSCALE   0.5\nOUTYSCALE   0.5\n"
        "OUTPOS      1.0 1.5\nNOUT        4 3\n")
    (tmp_path / "cfg").write_text(
        "PSFXSCALE   0.25\nPSFYSCALE   0.25\nNEXP        2\nUSERXY      0\n"
        "INCONFIG1   in1\nINCONFIG2   in2\nOUTCONFIG   out\n")
    prob = config.load_problem(str(tmp_path / "cfg"))
    assert (prob.n, prob.m, prob.n1out, prob.n2out) == (60, 12, 4, 3)
    xu, yu = problem.grid_xy(6, 5, [1.0, 1.0], [1.0, 1.0], [(0.0, 0.0), (0.25, -0.5)])
    assert np.array_equal(prob.x_i, xu.reshape(-1, order="F"))
    assert np.array_equal(prob.y_i, yu.reshape(-1, order="F"))
    Xa, Ya = problem.grid_XaYa(4, 3, 0.5, 0.5, 1.0, 1.5)
    assert np.array_equal(prob.X_a, Xa) and np.array_equal(prob.Y_a, Ya)
    # one PSF file with different rotations counts as constant (the reference's
    # imcom_test_psfconst quirk), so only the first exposure's PSF is used
    assert prob.psfconst == 1 and prob.nexppsf == 1
    assert np.array_equal(prob.noise, [2.0, 2.0])
    assert prob.meta["config"].cachefiles == {}


def test_missing_line_is_an_error(tmp_path):
    (tmp_path / "cfg").write_text("PSFXSCALE   0.25\nPSFYSCALE   0.25\n")
    with pytest.raises(config.ConfigError):
        config.read_config(str(tmp_path / "cfg"))
