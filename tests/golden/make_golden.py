"""Generate the committed golden fixtures ``tests/golden/*.npz``.

The reference ships no golden vectors for its solve path and cannot be
compiled here, so the fixtures come from ``numpy_mirror.py``, an independent
numpy/scipy restatement (pure-Python Neville, numpy FFT, scipy's LAPACK
DSYEVR driver).  Tests pin the C++ oracle and the GPU library against them.

Usage: ``python tests/golden/make_golden.py`` (about a minute).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from imcom_b200 import synth  # noqa: E402
import numpy_mirror  # noqa: E402

CASES = {
    # name: (workload, overrides, UnotS, US_max, tol, maxnits)
    "tiny_u": ("tiny", {}, True, 1e-4, 1e-7, 40),
    "tiny_s": ("tiny", {}, False, 0.25, 1e-4, 53),
    "tiny_rot": ("tiny", dict(rot_range=5.0, psf_kind="airy", psf_param=0.5), True, 2e-2, 1e-5, 53),
}

INPUT_KEYS = ("x_i", "y_i", "exp_i", "I_i", "X_a", "Y_a", "G_unrot", "Gamma", "rotangdeg", "noise")
OUTPUT_KEYS = ("C", "A", "B", "L", "K", "US", "nevals", "T", "H", "S", "U", "kappa_min",
               "kappa_max")


def problem_from(d):
    from imcom_b200.problem import Problem
    return Problem(x_i=d["x_i"], y_i=d["y_i"], exp_i=d["exp_i"].astype(np.int32), I_i=d["I_i"],
                   X_a=d["X_a"], Y_a=d["Y_a"], n1out=int(d["n1out"]), n2out=int(d["n2out"]),
                   G_unrot=np.asfortranarray(d["G_unrot"]), Gamma=np.asfortranarray(d["Gamma"]),
                   rotangdeg=d["rotangdeg"], noise=d["noise"], psfxscale=float(d["psfxscale"]),
                   psfyscale=float(d["psfyscale"]), psfconst=int(d["psfconst"]))


def load(name):
    d = dict(np.load(os.path.join(HERE, name + ".npz")))
    return problem_from(d), d


def main():
    for name, (wl, over, UnotS, US, tol, maxnits) in CASES.items():
        prob = synth.make(wl, seed=0, **over)
        out = numpy_mirror.solve(prob, UnotS=UnotS, US=US, tol=tol, maxnits=maxnits)
        rec = {k: getattr(prob, k) for k in INPUT_KEYS}
        rec.update(n1out=prob.n1out, n2out=prob.n2out, psfxscale=prob.psfxscale,
                   psfyscale=prob.psfyscale, psfconst=prob.psfconst, UnotS=int(UnotS),
                   US_max=US, tol=tol, maxnits=maxnits)
        rec.update({k: out[k] for k in OUTPUT_KEYS})
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
        print(name, "n", prob.n, "m", prob.m, "nps", prob.nps, "nevals",
              np.percentile(out["nevals"], [0, 50, 100]))


if __name__ == "__main__":
    main()
