"""IMCOM configuration files -> an in-memory ``Problem``.

Restates what the reference's driver does before the solve path starts, so a
configuration written for the reference (for example its own
``example/userxy1/config_example``) reaches this library's solve path with the
same inputs the Fortran driver would hand it:

* ``imcom_read_config`` (imcom_io.f90:499-677): PSFXSCALE, PSFYSCALE, NEXP,
  USERXY, one INCONFIG line per exposure, OUTCONFIG, then optional
  AFILE/BFILE/QFILE/LFILE/PFILE cache names;
* ``imcom_read_inconfigs`` (imcom_io.f90:681-825): PSFFILE, GIMFILE,
  ROTANGDEG, NOISE, then GIMXFILE/GIMYFILE (USERXY = 1) or GIMXSCALE,
  GIMYSCALE, DITHER (USERXY = 0);
* ``imcom_read_outconfig`` (imcom_io.f90:829-971): GAMFILE, OUTFILE, KFILE,
  TFILE, SFILE, UFILE, then OUTXFILE/OUTYFILE or OUTXSCALE, OUTYSCALE, OUTPOS,
  NOUT;
* then imcom.f90:56-84: the images and their mask (``imcom_alloc_gims``,
  saturation = the command line's 7th argument, DLAMCH('O') by default), the
  coordinates read (``imcom_alloc_xy``, ``imcom_alloc_XaYa``) or built
  (``imcom_build_xy``, ``imcom_build_XaYa``), ``imcom_test_psfconst`` and the
  padded, normalised PSFs (``imcom_alloc_psfs``).

Lines whose value is a file name are read as the reference reads them
(``FMT='(A12, A)'``: a 12-character keyword field, then the name, blanks
trimmed); numeric lines are list-directed (a keyword, then the values).
Relative file names are taken relative to the directory of the main
configuration file (the reference opens them relative to its working
directory, which is that directory in its documented usage).  Images are read
with this library's FITS reader (``imcom_b200.fits``).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

from . import fits
from .problem import (Problem, choose_npsf, grid_XaYa, grid_xy, mask_images, pad_psf,
                      test_psfconst)

DBL_MAX = np.finfo(np.float64).max  # DLAMCH('O'), the reference's default saturation


class ConfigError(ValueError):
    """A configuration line the reference would stop on."""


def _name_line(line: str) -> str:
    """FMT='(A12, A)': the value is everything after column 12, trimmed."""
    return line[12:].strip() if len(line) > 12 else ""


def _values(line: str, count: int, kind=float):
    toks = line.replace(",", " ").split()
    if len(toks) < count + 1:
        raise ConfigError(f"expected a keyword and {count} value(s): {line!r}")
    conv = (lambda t: float(t.replace("d", "e").replace("D", "e"))) if kind is float else int
    vals = [conv(t) for t in toks[1:count + 1]]
    return vals[0] if count == 1 else vals


@dataclass
class Config:
    """The settings of one IMCOM configuration (imcom_data.f90 names)."""

    directory: str
    psfxscale: float
    psfyscale: float
    nexp: int
    userxy: int
    psffile: list
    gimfile: list
    rotangdeg: list
    noise: list
    gimxfile: list = field(default_factory=list)
    gimyfile: list = field(default_factory=list)
    gimxscale: list = field(default_factory=list)
    gimyscale: list = field(default_factory=list)
    dither: list = field(default_factory=list)
    gamfile: str = ""
    outfiles: dict = field(default_factory=dict)   # H, K, T, S, U map file names
    outxfile: str = ""
    outyfile: str = ""
    outxscale: float = 0.0
    outyscale: float = 0.0
    outpos: tuple = (0.0, 0.0)
    nout: tuple = (0, 0)
    cachefiles: dict = field(default_factory=dict)  # A, B, Q, L, P cache file names

    def path(self, name: str) -> str:
        return name if os.path.isabs(name) else os.path.join(self.directory, name)


def read_config(path: str) -> Config:
    """Parse a main configuration file and the input/output files it names."""
    directory = os.path.dirname(os.path.abspath(path))
    lines = [ln.rstrip("\n") for ln in open(path)]
    it = iter(lines)

    def nxt(what):
        try:
            return next(it)
        except StopIteration:
            raise ConfigError(f"{path}: end of file before {what}") from None

    psfx = _values(nxt("PSFXSCALE"), 1)
    psfy = _values(nxt("PSFYSCALE"), 1)
    nexp = _values(nxt("NEXP"), 1, int)
    userxy = _values(nxt("USERXY"), 1, int)
    inconfig = [_name_line(nxt("INCONFIG")) for _ in range(nexp)]
    cfg = Config(directory=directory, psfxscale=psfx, psfyscale=psfy, nexp=nexp, userxy=userxy,
                 psffile=[], gimfile=[], rotangdeg=[], noise=[])
    for name in inconfig:
        sub = [ln.rstrip("\n") for ln in open(cfg.path(name))]
        need = 6 if userxy == 1 else 7
        if len(sub) < need:
            raise ConfigError(f"{name}: expected {need} lines")
        cfg.psffile.append(_name_line(sub[0]))
        cfg.gimfile.append(_name_line(sub[1]))
        cfg.rotangdeg.append(_values(sub[2], 1))
        cfg.noise.append(_values(sub[3], 1))
        if userxy == 1:
            cfg.gimxfile.append(_name_line(sub[4]))
            cfg.gimyfile.append(_name_line(sub[5]))
        else:
            cfg.gimxscale.append(_values(sub[4], 1))
            cfg.gimyscale.append(_values(sub[5], 1))
            cfg.dither.append(tuple(_values(sub[6], 2)))
    outconfig = _name_line(nxt("OUTCONFIG"))
    out = [ln.rstrip("\n") for ln in open(cfg.path(outconfig))]
    need = 8 if userxy == 1 else 10
    if len(out) < need:
        raise ConfigError(f"{outconfig}: expected {need} lines")
    cfg.gamfile = _name_line(out[0])
    cfg.outfiles = {k: _name_line(out[i]) for i, k in enumerate("HKTSU", start=1)}
    if userxy == 1:
        cfg.outxfile, cfg.outyfile = _name_line(out[6]), _name_line(out[7])
    else:
        cfg.outxscale = _values(out[6], 1)
        cfg.outyscale = _values(out[7], 1)
        cfg.outpos = tuple(_values(out[8], 2))
        cfg.nout = tuple(_values(out[9], 2, int))
    # optional cache names; the reference falls back to its defaults at EOF
    for key in "ABQLP":
        try:
            ln = next(it)
        except StopIteration:
            break
        cfg.cachefiles[key] = _name_line(ln)
    return cfg


def load_problem(path: str, saturation: float = DBL_MAX, name: str | None = None) -> Problem:
    """The solve path's inputs for the configuration at `path`, as the
    reference driver assembles them (imcom.f90:56-84)."""
    cfg = read_config(path)
    images = [fits.read(cfg.path(f)) for f in cfg.gimfile]
    shape = images[0].shape
    if any(im.shape != shape for im in images):
        raise ConfigError("variable size input images are not supported (imcom_alloc_gims)")
    ims = np.stack(images, axis=2)
    I_i, exp_i, subs = mask_images(np.asfortranarray(ims), saturation)
    if cfg.userxy == 1:
        xu = np.stack([fits.read(cfg.path(f), shape) for f in cfg.gimxfile], axis=2)
        yu = np.stack([fits.read(cfg.path(f), shape) for f in cfg.gimyfile], axis=2)
        Xa = fits.read(cfg.path(cfg.outxfile))
        Ya = fits.read(cfg.path(cfg.outyfile), Xa.shape)
        n1out, n2out = Xa.shape
        X_a, Y_a = Xa.reshape(-1, order="F").copy(), Ya.reshape(-1, order="F").copy()
    else:
        xu, yu = grid_xy(shape[0], shape[1], cfg.gimxscale, cfg.gimyscale, cfg.dither)
        n1out, n2out = cfg.nout
        X_a, Y_a = grid_XaYa(n1out, n2out, cfg.outxscale, cfg.outyscale, *cfg.outpos)
    x_i = xu.reshape(-1, order="F")[subs].copy()
    y_i = yu.reshape(-1, order="F")[subs].copy()
    psfconst = test_psfconst(cfg.psffile, cfg.rotangdeg)
    nexppsf = 1 if psfconst else cfg.nexp
    stamps = [fits.read(cfg.path(f)) for f in cfg.psffile[:nexppsf]]
    gam = fits.read(cfg.path(cfg.gamfile))
    if any(s.shape != stamps[0].shape for s in stamps) or gam.shape != stamps[0].shape:
        raise ConfigError("variable size PSF images are not supported (imcom_alloc_psfs)")
    nps = choose_npsf(x_i, y_i, X_a, Y_a, cfg.psfxscale, cfg.psfyscale, stamps[0].shape)
    G = np.zeros((nps, nps, nexppsf), order="F")
    for e, s in enumerate(stamps):
        G[:, :, e] = pad_psf(s, nps)
    return Problem(x_i=x_i, y_i=y_i, exp_i=exp_i, I_i=I_i, X_a=X_a, Y_a=Y_a, n1out=n1out,
                   n2out=n2out, G_unrot=G, Gamma=pad_psf(gam, nps),
                   rotangdeg=np.asarray(cfg.rotangdeg, dtype=np.float64),
                   noise=np.asarray(cfg.noise, dtype=np.float64), psfxscale=cfg.psfxscale,
                   psfyscale=cfg.psfyscale, psfconst=psfconst,
                   name=name or os.path.basename(path), meta={"config": cfg})
