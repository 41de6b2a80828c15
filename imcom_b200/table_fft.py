"""The lookup tables' inverse FFT: the library's own pruned, fused transform
(IMCOM_OPT_TABLE_FFT = 1, csrc/table_fft.cu: the register path at nps = 576,
the Stockham path at other sides) against embedding + cuFFT + shift, on one
workload.  By default (IMCOM_TABLE_FFT_AUTO) the library takes the register
path where it applies and cuFFT elsewhere.

    python -m imcom_b200.table_fft [--workload n4096] [--reps 5]

prints one JSON line: per path the median table-build time of the A tables
(E(E+1)/2 of them) and the B tables (E) from imcom_gpu_table_times (CUDA
events around the build on the library stream), the largest difference of
A and B between the paths relative to their largest entry, and the own
path's algorithmic HBM bytes per build (pass 1 writes and pass 2 reads the
nps x L intermediate, pass 2 writes the L x L table) against the measured
copy bandwidth.
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np

from . import synth
from .api import OPT_TABLE_FFT, TABLE_FFT_CUFFT, TABLE_FFT_OWN, Solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback 6.65 TB/s"


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def measure(workload="n4096", reps=5, device=0, seed=0):
    prob = synth.make(workload, seed)
    nps, E = prob.nps, prob.nexppsf
    L = 3 * nps
    out = {"workload": workload, "nps": nps, "side": L, "A_tables": E * (E + 1) // 2,
           "B_tables": E, "reps": reps}
    mats = {}
    for name, mode in (("cufft", TABLE_FFT_CUFFT), ("own", TABLE_FFT_OWN)):
        with Solver(device) as s:
            s.set_option(OPT_TABLE_FFT, mode)
            s.set_problem(prob)
            s.psf_spectra()
            A = s.build_A()
            B = s.build_B()
            mats[name] = (A, B)
            ta, tb = [], []
            for _ in range(reps):
                s.build_A(out=False)
                s.build_B(out=False)
                t = s.table_times()
                ta.append(t["A_tables"])
                tb.append(t["B_tables"])
            out[name] = {"A_tables_ms": float(np.median(ta)), "B_tables_ms": float(np.median(tb)),
                         "build_A_ms": s.stage_times()["build_A"],
                         "build_B_ms": s.stage_times()["build_B"]}
    (A0, B0), (A1, B1) = mats["cufft"], mats["own"]
    out["max_rel_diff_A"] = _rel(A1, A0)
    out["max_rel_diff_B"] = _rel(B1, B0)
    hbm, src = _hbm_peak()
    per_table = 32.0 * nps * L + 8.0 * L * L
    for kind, ntab in (("A", E * (E + 1) // 2), ("B", E)):
        t = out["own"][f"{kind}_tables_ms"] * 1e-3
        if t > 0:
            gbs = per_table * ntab / t / 1e9
            out["own"][f"{kind}_roofline"] = {"bound": "hbm", "algorithmic_bytes": per_table * ntab,
                                              "achieved_gbs": gbs, "peak": hbm,
                                              "peak_source": src, "frac": gbs / hbm}
        t0 = out["cufft"][f"{kind}_tables_ms"]
        out[f"speedup_{kind}_tables"] = t0 / out["own"][f"{kind}_tables_ms"] if t > 0 else None
    return out


def main():
    ap = argparse.ArgumentParser(description="lookup-table inverse FFT: own vs cuFFT")
    ap.add_argument("--workload", default="n4096")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    print(json.dumps(measure(args.workload, args.reps, args.device)), flush=True)


if __name__ == "__main__":
    main()
