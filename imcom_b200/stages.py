"""Run one solve of a synthetic workload stage by stage and print the GPU time
of every stage (CUDA events inside the library).  Each stage sits in an NVTX
range named after it (SPECTRA, A, EIG, B, P, BISECT, T, EPI), so a profiler
can select one stage's kernels, e.g.

    ncu --nvtx --nvtx-include "P/" -k regex:dgemm_kernel -c 1 \\
        python -m imcom_b200.stages n4096

Usage: python -m imcom_b200.stages [workload] [--library-eigensolver] [--twostage]
                                    [--split] [--learned] [--also-plain-bisect]
                                    [--table-features] [--own-table-fft]
                                    [--repeat-bisect N] [--stacks S] [--stop-after STAGE]
       python -m imcom_b200.stages jacobi     (64 batched 112 x 112 Jacobi eigensolves)
       python -m imcom_b200.stages train      (features of the small workload, 2 epochs)

--twostage        the two-stage eigensolver (IMCOM_EIGH_TWOSTAGE)
--also-plain-bisect  with --learned, run the plain bisection first as well
--stacks S        after the solve, H = T^T I for S random image stacks with the
                  streaming kernel (IMCOM_OPT_STACK_KERNEL = 1)
--stop-after STAGE  stop after SPECTRA, A, EIG, B, P, BISECT or T

--split           P and T on the split-precision int8 product (IMCOM_PREC_SPLIT)
--learned         learned-kappa bracket (committed weights) instead of the plain
                  bisection
--table-features  learned-kappa features from the neighbour table and band
                  segments (IMCOM_OPT_KAPPA_FEATURES = 1)
--own-table-fft   the library's own inverse FFT for the lookup tables at every
                  side it covers (IMCOM_OPT_TABLE_FFT = 1; default 2: own
                  where faster than cuFFT)
--repeat-bisect N run the bisection N more times and print each one's time
--compare-features  after the solve, time 5 learned bisections with the scanned
                  features and 5 with the table-built ones (committed weights),
                  check that K is identical, and print one JSON line
"""
from __future__ import annotations

import json
import sys


def run_stages(s, stage, learned, argv, out):
    """The solve, stage by stage (each stage in its NVTX range)."""
    from . import EPS
    C = stage("SPECTRA", lambda: s.psf_spectra())
    out["C"] = C
    stage("A", lambda: s.build_A(out=False))
    stage("EIG", lambda: s.eigen_A(out=False))
    stage("B", lambda: s.build_B(out=False))
    stage("P", lambda: s.build_P(out=False))
    if learned and "--also-plain-bisect" in argv:
        stage("BISECT", lambda: s.bisect_kappa(True, 1e-2, C * EPS, C / EPS, 1e-5, 53, C,
                                               out=False))
    if learned:
        stage("BISECT", lambda: s.bisect_kappa_learned(True, 1e-2, C * EPS, C / EPS, 1e-5, 53,
                                                       C, out=False))
    else:
        stage("BISECT", lambda: s.bisect_kappa(True, 1e-2, C * EPS, C / EPS, 1e-5, 53, C,
                                               out=False))
    stage("T", lambda: s.build_T(out=False))
    stage("EPI", lambda: (s.build_S(out=False), s.build_image(out=False)))


def extra_case(wl):
    """The cases that are not one solve: batched Jacobi and MLP training."""
    import numpy as np

    from . import Solver, synth
    with Solver(0) as s:
        if wl == "jacobi":
            rng = np.random.default_rng(0)
            A = rng.standard_normal((64, 112, 112))
            _, L, sweeps = s.eigh_jacobi_batched(A @ np.transpose(A, (0, 2, 1)))
            print({"matrices": 64, "n": 112, "max_sweeps": int(sweeps.max())})
        else:
            from .kappa_model import collect, train
            feat, y = collect(s, [synth.make("small", 0)], [1e-2])
            train(s, feat, y, epochs=2)
            print({"samples": int(y.size)})


def main(argv):
    import torch

    from . import EIGH_DC, EIGH_LIBRARY, EIGH_TWOSTAGE, EPS, Solver, synth
    from .api import OPT_KAPPA_FEATURES, OPT_STACK_KERNEL, OPT_TABLE_FFT

    wl = argv[0] if argv and not argv[0].startswith("-") else "n4096"
    if wl in ("jacobi", "train"):
        return extra_case(wl)
    stop = argv[argv.index("--stop-after") + 1] if "--stop-after" in argv else None
    nv = torch.cuda.nvtx
    prob = synth.make(wl, 0)
    with Solver(0) as s:
        s.set_eigensolver(EIGH_LIBRARY if "--library-eigensolver" in argv else
                          EIGH_TWOSTAGE if "--twostage" in argv else EIGH_DC)
        s.set_precision("--split" in argv)
        s.set_option(OPT_KAPPA_FEATURES, 1 if "--table-features" in argv else 0)
        s.set_option(OPT_TABLE_FFT, 1 if "--own-table-fft" in argv else 2)
        compare = "--compare-features" in argv
        learned = "--learned" in argv or compare
        if learned:
            from .kappa_model import DEFAULT_WEIGHTS, KappaModel
            KappaModel.load(DEFAULT_WEIGHTS).install(s)
        s.set_problem(prob)

        class Stop(Exception):
            pass

        def stage(name, fn):
            nv.range_push(name)
            r = fn()
            s.synchronize()
            nv.range_pop()
            if name == stop:
                raise Stop
            return r

        C_holder = {}
        try:
            run_stages(s, stage, learned, argv, C_holder)
        except Stop:
            pass
        print({k: round(v, 3) for k, v in s.stage_times().items()})
        if stop is not None:
            return
        C = C_holder["C"]
        print({k: round(v, 3) for k, v in s.table_times().items()})
        if "--stacks" in argv:
            import numpy as np
            S = int(argv[argv.index("--stacks") + 1])
            s.set_option(OPT_STACK_KERNEL, 1)
            s.build_images(np.random.default_rng(0).standard_normal((prob.n, S)))
            s.set_option(OPT_STACK_KERNEL, 0)

        def bisect():
            if learned:
                return s.bisect_kappa_learned(True, 1e-2, C * EPS, C / EPS, 1e-5, 53, C,
                                              out=False)
            return s.bisect_kappa(True, 1e-2, C * EPS, C / EPS, 1e-5, 53, C, out=False)

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
