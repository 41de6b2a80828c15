"""Run one solve of a synthetic workload stage by stage and print the GPU time
of every stage (CUDA events inside the library).  Each stage sits in an NVTX
range named after it (SPECTRA, A, EIG, B, P, BISECT, T, EPI), so a profiler
can select one stage's kernels, e.g.

    ncu --nvtx --nvtx-include "P/" -k regex:dgemm_kernel -c 1 \\
        python -m imcom_b200.stages n4096

Usage: python -m imcom_b200.stages [workload] [--library-eigensolver] [--split]
                                    [--learned] [--table-features]
                                    [--own-table-fft] [--repeat-bisect N]

--split           P and T on the split-precision int8 product (IMCOM_PREC_SPLIT)
--learned         learned-kappa bracket (committed weights) instead of the plain
                  bisection
--table-features  learned-kappa features from the neighbour table and band
                  segments (IMCOM_OPT_KAPPA_FEATURES = 1)
--own-table-fft   the library's own inverse FFT for the lookup tables
                  (IMCOM_OPT_TABLE_FFT = 1)
--repeat-bisect N run the bisection N more times and print each one's time
--compare-features  after the solve, time 5 learned bisections with the scanned
                  features and 5 with the table-built ones (committed weights),
                  check that K is identical, and print one JSON line
"""
from __future__ import annotations

import json
import sys


def main(argv):
    import torch

    from . import EIGH_DC, EIGH_LIBRARY, EPS, Solver, synth
    from .api import OPT_KAPPA_FEATURES, OPT_TABLE_FFT

    wl = argv[0] if argv and not argv[0].startswith("-") else "n4096"
    nv = torch.cuda.nvtx
    prob = synth.make(wl, 0)
    with Solver(0) as s:
        s.set_eigensolver(EIGH_LIBRARY if "--library-eigensolver" in argv else EIGH_DC)
        s.set_precision("--split" in argv)
        s.set_option(OPT_KAPPA_FEATURES, 1 if "--table-features" in argv else 0)
        s.set_option(OPT_TABLE_FFT, 1 if "--own-table-fft" in argv else 0)
        compare = "--compare-features" in argv
        learned = "--learned" in argv or compare
        if learned:
            from .kappa_model import DEFAULT_WEIGHTS, KappaModel
            KappaModel.load(DEFAULT_WEIGHTS).install(s)
        s.set_problem(prob)

        def stage(name, fn):
            nv.range_push(name)
            r = fn()
            s.synchronize()
            nv.range_pop()
            return r

        C = stage("SPECTRA", lambda: s.psf_spectra())
        stage("A", lambda: s.build_A(out=False))
        stage("EIG", lambda: s.eigen_A(out=False))
        stage("B", lambda: s.build_B(out=False))
        stage("P", lambda: s.build_P(out=False))
        def bisect():
            if learned:
                return s.bisect_kappa_learned(True, 1e-2, C * EPS, C / EPS, 1e-5, 53, C,
                                              out=False)
            return s.bisect_kappa(True, 1e-2, C * EPS, C / EPS, 1e-5, 53, C, out=False)

        stage("BISECT", bisect)
        stage("T", lambda: s.build_T(out=False))
        stage("EPI", lambda: (s.build_S(out=False), s.build_image(out=False)))
        print({k: round(v, 3) for k, v in s.stage_times().items()})
        print({k: round(v, 3) for k, v in s.table_times().items()})
        if "--repeat-bisect" in argv:
            reps = int(argv[argv.index("--repeat-bisect") + 1])
            times = []
            for _ in range(reps):
                stage("BISECT", bisect)
                times.append(round(s.stage_times()["bisect"], 3))
            print({"bisect_ms": times})
        if compare:
            out = {"workload": wl}
            K = {}
            for name, mode in (("scan", 0), ("table", 1)):
                s.set_option(OPT_KAPPA_FEATURES, mode)
                K[name] = s.bisect_kappa_learned(True, 1e-2, C * EPS, C / EPS, 1e-5, 53, C)[0]
                times = []
                for _ in range(5):
                    stage("BISECT", bisect)
                    times.append(s.stage_times()["bisect"])
                out[f"bisect_ms_{name}"] = sorted(times)[2]
            out["K_identical"] = bool((K["scan"] == K["table"]).all())
            out["speedup"] = out["bisect_ms_scan"] / out["bisect_ms_table"]
            print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
