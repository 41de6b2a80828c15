#!/usr/bin/env python
"""Benchmark: output pixels/s of the IMCOM solve path at n=4096.

A step is one full solve of the n=4096 workload (4 exposures of 32x32 input
pixels with U[-5,5] deg rotations and uniform dithers, Airy lambda/D = 0.5 px
(x) pixel PSFs, Gamma Gaussian sigma = 0.9 px, 64x64 output at 0.5 px,
lookup side 1728): PSF spectra -> A tables + assembly -> eigendecomposition
-> B tables + assembly -> P -> per-pixel kappa bisection (U < 1e-2, tolerance
1e-5) -> T -> S and H.  Synthetic seeded inputs (synth.make("n4096")).

Two forms of the path are timed on the same workload and tolerance:
  plain  FP64 P and T (DMMA) and the plain bisection;
  fast   learned-kappa bracket and split-precision P and T (int8 digit slices
         on the tcgen05 tensor cores, audited, FP64 recomputation of the
         pixels that fail the audit) -- the headline `value`.
Each is timed as the full solve and as the cached-system stage (P -> kappa ->
T -> S, H with Q, L and B resident, the reference's cached path), at the
headline target and again at a strict one (``strict_target``: U < 1e-6,
tolerance 1e-8).

  value  fast full-solve pixels/s with the inputs resident in HBM (no host
         copies timed), CUDA events on the library's stream, L2 flushed
         between steps.
  e2e    the same metric through the C-ABI with pinned host buffers: inputs
         copied in and H, K, U, S and T copied out inside every step.

``batch``: the batched-patch workload -- 256 independent patches of uneven n
(990-2270, masked pixels) solved by a pool of contexts per GPU, each on a
share of the SMs, concurrency chosen by the autotuner; with N GPUs the
patches are split across ranks by cost (no data-path collective); patches/s
and output pixels/s over the slowest rank's wall-clock time.

``t_reuse``: T reused for many image stacks -- H = T^T I for 1, 8, 16 and 64
stacks at once with T resident (imcom_b200/t_reuse.py), through the FP64 GEMM
and through the streaming kernel, each in a child process after the timed
solves.  ``table_fft``: the n=4096 lookup tables' inverse FFT through the
library's own pruned, fused transform against embedding + cuFFT + shift
(imcom_b200/table_fft.py), in a child process too.  ``kappa_features``: the
learned bisection with its features scanned per pixel against the neighbour
table and band segments (python -m imcom_b200.stages --compare-features).

``--impl reference`` times the CPU oracle (the reference's algorithm restated
in C++ with OpenMP + LAPACK/BLAS) on the same workload, all host cores.
Multi-GPU (``torchrun``): replicas only -- every rank solves its own
independent patch (seed = rank); value = all ranks' pixels / max rank time.
"""
from __future__ import annotations

import argparse
import faulthandler
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "n4096"
UNOTS, US_MAX, US_TOL, MAXNITS = True, 1e-2, 1e-5, 53
STRICT = (1e-6, 1e-8)  # the strict leakage target reported beside the headline one
METRIC = "output pixels/s at n=4096 (learned-κ+mixed vs plain FP64 GPU, same U/Σ tol)"
UNIT = "pixels/s"
# the same string on both arms' lines
WORKLOAD_DESC = ("n4096: 4x32x32 inputs (n=4096), rotations U[-5,5] deg, Airy lambda/D=0.5 px "
                 "PSF, 64x64 output at 0.5 px (m=4096), U mode U<1e-2 tol 1e-5, maxnits 53")
L2_BYTES = 126 * 1024 * 1024


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def int8_gemm_peak(torch, dev):
    """cuBLAS int8 GEMM throughput (TOP/s, torch._int_mm, 8192^3) measured
    here: the denominator of the split product's tensor roofline."""
    n = 8192
    a = torch.randint(-128, 127, (n, n), dtype=torch.int8, device=dev)
    b = torch.randint(-128, 127, (n, n), dtype=torch.int8, device=dev)
    for _ in range(2):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def pinned_like(torch, arr):
    """Copy a numpy array into page-locked host memory (same layout)."""
    arr = np.asarray(arr)
    if arr.ndim <= 1 or arr.flags.c_contiguous and not arr.flags.f_contiguous:
        t = torch.empty(arr.shape, dtype=getattr(torch, str(arr.dtype)), pin_memory=True)
        out = t.numpy()
        out[...] = arr
        return out, t
    t = torch.empty(arr.shape[::-1], dtype=getattr(torch, str(arr.dtype)), pin_memory=True)
    out = t.numpy().T  # Fortran-contiguous view
    out[...] = arr
    return out, t


def cpu_baseline(prob, steps=1):
    from oracle import oracle as O
    t = []
    for _ in range(steps):
        t0 = time.perf_counter()
        O.solve(prob, UnotS=UNOTS, US_max=US_MAX, US_tol=US_TOL, maxnits=MAXNITS,
                keep_tables=False)
        t.append(time.perf_counter() - t0)
    return t, O.get_threads()


BATCH_KW = dict(UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=40)


def batched_patches(npatch=256, sample=48, rank=0, world=1, dist=None, device=None, repeats=5,
                    cpu_sample=8):
    """The batched-patch workload: `npatch` patches of 4 exposures of side
    U{16..24} with 2% of input pixels masked (n ~ 990-2270), per-exposure
    Gaussian PSF sigma ~ U[0.5, 0.8] px, 24x24 outputs; U < 1e-6, tolerance
    1e-8, 40 iterations.  With several ranks every rank solves its share of the
    same `npatch` patches (balanced by n^3, no data-path collective).  Each
    rank's concurrency (contexts side by side, each on a share of the SMs) is
    chosen by the autotuner on the first `sample` of its patches, together
    with the cluster that finishes each tridiagonalisation; its patches are
    then solved once to plan every FFT size and once timed (wall clock around
    the pool, results copied to the host); the job's time is the slowest
    rank's."""
    from imcom_b200 import batch, replicas
    problems = batch.make_batch(npatch, seed0=1000)
    mine = replicas.shard_by_cost([replicas.patch_cost(p) for p in problems], rank, world)
    local = [problems[i] for i in mine]
    if local:
        tune = batch.autotune(local[:sample], candidates=(1, 2, 3, 4, 6, 8), tails=(0, 8, -1),
                              **BATCH_KW)
    else:  # more ranks than patches: this rank only joins the barrier and the MAX
        tune = batch.Tuning(1, 0, {})
    k = tune.concurrency
    times = []
    with batch.BatchSolver(k, tail_ctas=tune.tail_ctas) as b:
        if local:
            b.solve(local, **BATCH_KW)
        for _ in range(repeats):
            if dist is not None:
                dist.barrier()
            r = b.solve(local, **BATCH_KW) if local else batch.BatchResult(concurrency=k)
            times.append(replicas.max_over_ranks(r.seconds, dist, device))
    t = statistics.median(times)
    ns = [p.n for p in problems]
    out = {"workload": f"{npatch} patches, 4 exposures of side U{{16..24}}, 2% masked, "
                       "24x24 outputs, U<1e-6 tol 1e-8",
           "n_range": [min(ns), max(ns)], "psf_sides": len({p.nps for p in problems}),
           "patches_per_s": replicas.job_rate(npatch, t),
           "pixels_per_s": replicas.job_rate(sum(p.m for p in problems), t),
           "seconds": t, "runs": len(times),
           "patches_per_s_runs": [replicas.job_rate(npatch, x) for x in times],
           "spread": (max(times) - min(times)) / t if times else None,
           "ranks": world, "patches_rank0": len(local),
           "concurrency": k, "sm_share": r.sm_share, "tail_ctas": tune.tail_ctas,
           "autotune_patches_per_s": {f"{q}x{'auto' if tt == 0 else ('none' if tt < 0 else tt)}": v
                                      for (q, tt), v in tune.rates.items()},
           "timing": f"median of {len(times)} timed passes, wall clock around each rank's "
                     "thread pool after one warm pass, max over ranks"}
    if rank == 0 and cpu_sample > 0:
        # the oracle on every (npatch / cpu_sample)-th patch: sizes across the range
        from oracle import oracle as O
        pick = sorted(range(npatch), key=lambda i: problems[i].n)[::max(1, npatch // cpu_sample)]
        t0 = time.perf_counter()
        for i in pick:
            O.solve(problems[i], keep_tables=False, **BATCH_KW)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": len(pick) / dt, "unit": "patches/s",
                               "cores": O.get_threads(), "kind": "port",
                               "sample": f"{len(pick)} of the {npatch} patches (every "
                                         f"{max(1, npatch // cpu_sample)}th by size, n "
                                         f"{problems[pick[0]].n}-{problems[pick[-1]].n}) "
                                         "through the C++ restatement, OpenMP + OpenBLAS"}
    return out


def child_measure(module, *args, timeout=300):
    """Run `python -m <module> <args>` (a measurement that prints one JSON
    line) in a child process with its own CUDA context, so this line keeps
    its other numbers whatever that run meets; returns its JSON or an
    {"error": ...} object."""
    try:
        r = subprocess.run([sys.executable, "-m", module, *args], cwd=ROOT,
                           capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"error": f"no result within {timeout} s"}
    lines = r.stdout.strip().splitlines()
    if r.returncode != 0 or not lines:
        tail = (r.stderr or r.stdout).strip().splitlines()[-3:]
        return {"error": f"exit {r.returncode}: " + " | ".join(tail)}
    try:
        return json.loads(lines[-1])
    except ValueError:
        return {"error": "unreadable output: " + lines[-1][:200]}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    from imcom_b200 import synth
    prob = synth.make(WORKLOAD, seed=0)
    cpu_baseline(prob, steps=args.warmup)
    times, cores = cpu_baseline(prob, steps=args.steps)
    v = prob.m / statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC, "n": prob.n, "m": prob.m,
                   "nps": prob.nps, "lookup_side": 3 * prob.nps},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": "one full n=4096 solve per step (C++ restatement of the "
                                   "reference, OpenMP + OpenBLAS LAPACK/BLAS)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
    from imcom_b200 import EIGH_DC, EIGH_LIBRARY, Solver, synth
    from imcom_b200.problem import build_Ndiag

    prob = synth.make(WORKLOAD, seed=rank)
    s = Solver(local)
    s.set_eigensolver(EIGH_LIBRARY if args.eigensolver == "library" else EIGH_DC)
    stream = torch.cuda.ExternalStream(s.stream(), device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    Nd = build_Ndiag(prob.n, prob.noise)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    learned = args.kappa == "learned"
    split = args.precision == "split"
    EPS = 1.1102230246251565e-16

    def system():
        C = s.psf_spectra()
        s.build_A(out=False)
        s.eigen_A(out=False)
        s.build_B(out=False)
        return C

    def stage2(fast, C, out=False, us=US_MAX, tol=US_TOL):
        """P -> kappa -> T -> S, H on the resident system."""
        s.set_precision(fast and split)
        kmin, kmax = C * EPS, C / EPS
        r = {"P": s.build_P(out=out)}
        if fast and learned:
            r["K"], r["US"], r["nev"], _ = s.bisect_kappa_learned(UNOTS, us, kmin, kmax, tol,
                                                                  MAXNITS, C, out=out)
        else:
            r["K"], r["US"], r["nev"] = s.bisect_kappa(UNOTS, us, kmin, kmax, tol, MAXNITS, C,
                                                       out=out)
        r["T"] = s.build_T(out=out)
        r["S"] = s.build_S(out=out)
        r["H"] = s.build_image(out=out)
        return r

    def device_step(fast, us=US_MAX, tol=US_TOL):
        C = system()
        stage2(fast, C, us=us, tol=tol)

    # ---- learned-kappa model (trained outside the timed region) -------------
    model_src = None
    if learned:
        from imcom_b200 import kappa_model as KM
        if os.path.exists(KM.DEFAULT_WEIGHTS):
            model = KM.KappaModel.load(KM.DEFAULT_WEIGHTS)
            model_src = "committed weights " + os.path.basename(KM.DEFAULT_WEIGHTS)
        else:
            rng = np.random.default_rng(12345)
            probs = [synth.make(WORKLOAD, seed=1000 + q) for q in range(8)]
            targets = list(10.0 ** rng.uniform(np.log10(3e-3), np.log10(3e-2), len(probs)))
            feat, y = KM.collect(s, probs, targets)
            model, _ = KM.train(s, feat, y, epochs=40)
            model_src = f"trained at start-up on {y.size} pixels of 8 fresh seeds"
        model.install(s)

    # ---- value: inputs resident in HBM ------------------------------------
    s.set_problem(prob)

    def timed(fn, nsteps):
        for _ in range(args.warmup):
            fn()
        s.synchronize()
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        l0 = s.launch_count()
        st, sm = [], []
        for _ in range(nsteps):
            flush.fill_(1.0)  # evict L2 between timed steps
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            s.synchronize()
            sm.append(e0.elapsed_time(e1))
            st.append(s.stage_times())
        return sm, st, (s.launch_count() - l0) // max(1, nsteps)

    plain_ms, plain_st, _ = timed(lambda: device_step(False), args.steps)
    clocks = Clocks(local)
    clocks.start()
    step_ms, stage_ms, launches = timed(lambda: device_step(True), args.steps)
    torch.cuda.synchronize()
    ck = clocks.stop()
    barrier()
    t_step = max_over_ranks(statistics.mean(step_ms))
    t_plain = max_over_ranks(statistics.mean(plain_ms))
    value = world * prob.m / (t_step * 1e-3)
    plain_value = world * prob.m / (t_plain * 1e-3)

    # ---- cached-system stage: P -> kappa -> T -> S, H on resident Q, L, B ---
    C = system()
    c_plain, c_plain_st, _ = timed(lambda: stage2(False, C), args.steps)
    c_fast, c_fast_st, _ = timed(lambda: stage2(True, C), args.steps)
    tc_plain = max_over_ranks(statistics.mean(c_plain))
    tc_fast = max_over_ranks(statistics.mean(c_fast))
    cached = {"plain_fp64_value": world * prob.m / (tc_plain * 1e-3),
              "value": world * prob.m / (tc_fast * 1e-3),
              "ms_plain": tc_plain, "ms": tc_fast, "speedup_vs_plain_fp64": tc_plain / tc_fast,
              "stages_ms_plain": {k: statistics.mean(d[k] for d in c_plain_st)
                                  for k in ("build_P", "bisect", "build_T", "epilogue")},
              "stages_ms": {k: statistics.mean(d[k] for d in c_fast_st)
                            for k in ("build_P", "bisect", "build_T", "epilogue")}}

    def relmax(a, b):
        return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))

    # ---- the same comparisons at a strict leakage target (U < 1e-6) ----------
    strict = None
    if split or learned:
        su, stol = STRICT
        sc_plain, sc_plain_st, _ = timed(lambda: stage2(False, C, us=su, tol=stol), args.steps)
        sc_fast, sc_fast_st, _ = timed(lambda: stage2(True, C, us=su, tol=stol), args.steps)
        sf_plain, _, _ = timed(lambda: device_step(False, su, stol), args.steps)
        sf_fast, _, _ = timed(lambda: device_step(True, su, stol), args.steps)
        C = system()
        srp = stage2(False, C, out=True, us=su, tol=stol)
        srf = stage2(True, C, out=True, us=su, tol=stol)
        sinfo = s.split_info() if split else {}
        scolT = (np.linalg.norm(srf["T"] - srp["T"], axis=0) /
                 np.linalg.norm(srp["T"], axis=0))
        t_sc_plain = max_over_ranks(statistics.mean(sc_plain))
        t_sc_fast = max_over_ranks(statistics.mean(sc_fast))
        t_sf_plain = max_over_ranks(statistics.mean(sf_plain))
        t_sf_fast = max_over_ranks(statistics.mean(sf_fast))
        strict = {
            "target": f"U<{su:g} tol {stol:g}",
            "full_solve": {"plain_fp64_value": world * prob.m / (t_sf_plain * 1e-3),
                           "value": world * prob.m / (t_sf_fast * 1e-3),
                           "speedup_vs_plain_fp64": t_sf_plain / t_sf_fast},
            "cached_stage": {"ms_plain": t_sc_plain, "ms": t_sc_fast,
                             "speedup_vs_plain_fp64": t_sc_plain / t_sc_fast,
                             "stages_ms_plain": {k: statistics.mean(d[k] for d in sc_plain_st)
                                                 for k in ("build_P", "bisect", "build_T",
                                                           "epilogue")},
                             "stages_ms": {k: statistics.mean(d[k] for d in sc_fast_st)
                                           for k in ("build_P", "bisect", "build_T",
                                                     "epilogue")}},
            "accuracy_vs_plain_fp64": {
                "kappa_identical": bool(np.array_equal(srf["K"], srp["K"])),
                "U_max_rel": relmax(srf["US"], srp["US"]),
                "T_column_max_rel": float(scolT.max()),
                "split_audit": sinfo},
            "mean_evaluations_plain": float(np.mean(srp["nev"])),
            "mean_evaluations_fast": float(np.mean(srf["nev"])),
        }

    # ---- accuracy of the fast path against the plain FP64 path (same system)
    C = system()
    rp = stage2(False, C, out=True)
    rf = stage2(True, C, out=True)
    info = s.split_info() if split else {}
    s.set_precision(False)

    colT = np.linalg.norm(rf["T"] - rp["T"], axis=0) / np.linalg.norm(rp["T"], axis=0)
    accuracy = {
        "kappa_identical": bool(np.array_equal(rf["K"], rp["K"])),
        "U_max_rel": relmax(rf["US"], rp["US"]),
        "S_max_rel": relmax(rf["S"], rp["S"]),
        "T_column_max_rel": float(colT.max()),
        "H_rel_normwise": float(np.linalg.norm(rf["H"] - rp["H"]) / np.linalg.norm(rp["H"])),
        "P_rel_normwise": float(np.linalg.norm(rf["P"] - rp["P"]) / np.linalg.norm(rp["P"])),
        "bars": "kappa identical, U/S <= 1e-6 rel, T columns <= 1e-8 rel",
        "split_audit": info,
    }
    kappa_info = {"solver": ("network start, Newton steps, certified bisection replay" if learned
                             else "bisection"),
                  "mean_evaluations_plain": float(np.mean(rp["nev"])),
                  "mean_evaluations_fast": float(np.mean(rf["nev"])),
                  "model": model_src}
    if learned:
        s.build_P(out=False)  # FP64 P again (the split path's P is the resident one)
        K1, _, nev_l, fb = s.bisect_kappa_learned(UNOTS, US_MAX, C * EPS, C / EPS, US_TOL,
                                                  MAXNITS, C)
        # the same FP64 P for both bisections (the fast path's figure below also
        # carries the split product's audit)
        ms_l, ms_p = [], []
        for _ in range(5):
            s.bisect_kappa_learned(UNOTS, US_MAX, C * EPS, C / EPS, US_TOL, MAXNITS, C,
                                   out=False)
            ms_l.append(s.stage_times()["bisect"])
            s.bisect_kappa(UNOTS, US_MAX, C * EPS, C / EPS, US_TOL, MAXNITS, C, out=False)
            ms_p.append(s.stage_times()["bisect"])
        kappa_info.update({"mean_evaluations_learned_fp64P": float(np.mean(nev_l)),
                           "no_bound_fraction": float(np.mean(fb)),
                           "bisect_ms_plain": cached["stages_ms_plain"]["bisect"],
                           "bisect_ms_fast": cached["stages_ms"]["bisect"],
                           "bisect_ms_fast_includes": "split-product audit",
                           "fp64P_bisect_ms_plain": statistics.median(ms_p),
                           "fp64P_bisect_ms_learned": statistics.median(ms_l)})

    # ---- e2e: through the C-ABI with pinned host buffers -------------------
    keep = []
    host = {}
    for k in ("x_i", "y_i", "exp_i", "X_a", "Y_a", "I_i", "G_unrot", "Gamma", "rotangdeg"):
        host[k], t = pinned_like(torch, getattr(prob, k))
        keep.append(t)
    host["Nd"], t = pinned_like(torch, Nd)
    keep.append(t)
    outs = {}
    for k, shape in (("T", (prob.n, prob.m)), ("H", (prob.m,)), ("K", (prob.m,)),
                     ("U", (prob.m,)), ("S", (prob.m,))):
        outs[k], t = pinned_like(torch, np.zeros(shape, order="F"))
        keep.append(t)
    h2d = sum(host[k].nbytes for k in host)
    d2h = sum(outs[k].nbytes for k in outs)

    def e2e_step():
        s.set_inputs(host["x_i"], host["y_i"], host["exp_i"], host["X_a"], host["Y_a"],
                     host["I_i"], host["Nd"], prob.psfxscale, prob.psfyscale)
        s.set_psfs(host["G_unrot"], host["rotangdeg"], host["Gamma"], prob.psfconst)
        s.set_precision(split)
        C = s.psf_spectra()
        kmin, kmax = C * EPS, C / EPS
        s.build_A(out=False)
        s.eigen_A(out=False)
        s.build_B(out=False)
        s.build_P(out=False)
        if learned:
            s._call("imcom_gpu_bisect_kappa_learned", 1, US_MAX, kmin, kmax, US_TOL, MAXNITS, C,
                    outs["K"].ctypes.data, outs["U"].ctypes.data, None, None)
        else:
            s._call("imcom_gpu_bisect_kappa", 1, US_MAX, kmin, kmax, US_TOL, MAXNITS, C,
                    outs["K"].ctypes.data, outs["U"].ctypes.data, None)
        s._call("imcom_gpu_build_T", outs["T"].ctypes.data)
        s._call("imcom_gpu_build_S", outs["S"].ctypes.data)
        s._call("imcom_gpu_build_image", outs["H"].ctypes.data)

    for _ in range(min(args.warmup, 2)):
        e2e_step()
    barrier()
    torch.cuda.synchronize()
    e2e_ms = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2e_step()
        s.synchronize()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    barrier()
    t_e2e = max_over_ranks(statistics.mean(e2e_ms))
    e2e_value = world * prob.m / (t_e2e * 1e-3)

    s.set_precision(False)

    # ---- roofline of the dominant own kernel -------------------------------
    avg = {k: statistics.mean(d[k] for d in stage_ms) for k in stage_ms[0]}
    n, m = prob.n, prob.m
    peaks = measured_peaks()
    own = {k: v for k, v in avg.items()
           if not k.startswith("eig_") and not (k == "eigen_A" and args.eigensolver == "library")}
    dom = max(own, key=own.get)
    if dom == "eigen_A":
        # dominant kernel: the tridiagonalisation panel kernel, bound by streaming the
        # symmetric trailing matrix once per column: sum_j R_j (R_j + 1) / 2 doubles
        byts = 8.0 * sum(r * (r + 1) / 2.0 for r in range(1, n))
        t_ms = avg.get("eig_tridiag") or avg[dom]
        ach = byts / (t_ms * 1e-3) / 1e9
        pk = peaks.get("hbm_gbs", 6650.0)
        # DRAM bytes of the 108 panel launches of one tridiagonalisation at n = 4096
        # (profiles/trd_traffic_n4096.md): the trailing matrix stays in L2
        traffic = 3.024e9 if n == 4096 else None
        roof = {"kernel": "trd_panel_kernel (eigen_A tridiagonalisation)", "bound": "hbm",
                "achieved": ach, "peak": pk, "unit": "GB/s", "frac": ach / pk,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                "algorithmic_bytes": byts, "traffic": traffic,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum over all "
                                  "panel launches of one tridiagonalisation "
                                  "(profiles/trd_traffic_n4096.md)"}
    else:
        byts = {"build_A": 8.0 * n * n, "build_B": 8.0 * n * m}.get(dom, 8.0 * n * m)
        ach = byts / (avg[dom] * 1e-3) / 1e9
        pk = peaks.get("hbm_gbs", 6650.0)
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": pk, "unit": "GB/s",
                "frac": ach / pk, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                "traffic": None}
    # the split product (tensor-bound): P takes 7 slices (28 int8 products),
    # T 6 slices (21); algorithmic int8 ops = products x 2 n^2 m per stage
    # time of the stage (slicing, product, audit included)
    split_roof = None
    if split and rank == 0:
        i8 = int8_gemm_peak(torch, dev)
        sP, sT = int(info.get("slices_P", 7)), int(info.get("slices_T", 6))
        opsP = sP * (sP + 1) / 2 * 2.0 * n * n * m
        opsT = sT * (sT + 1) / 2 * 2.0 * n * n * m
        tP, tT = cached["stages_ms"]["build_P"], cached["stages_ms"]["build_T"]
        split_roof = {"bound": "tensor", "unit": "TOP/s (int8)", "peak": i8,
                      "peak_source": "cuBLAS int8 GEMM 8192^3 (torch._int_mm) in this run",
                      "build_P": {"achieved": opsP / (tP * 1e-3) / 1e12,
                                  "frac": opsP / (tP * 1e-3) / 1e12 / i8},
                      "build_T": {"achieved": opsT / (tT * 1e-3) / 1e12,
                                  "frac": opsT / (tT * 1e-3) / 1e12 / i8},
                      "fp64_equivalent_TFLOPs": {
                          "build_P": 2.0 * n * n * m / (tP * 1e-3) / 1e12,
                          "build_T": 2.0 * n * n * m / (tT * 1e-3) / 1e12}}

    s.close()
    batch_line = None
    if not args.no_batch:  # every rank takes part (its share of the patches)
        try:
            batch_line = batched_patches(rank=rank, world=world, dist=dist, device=dev)
        except Exception as exc:  # noqa: BLE001 - the solve line still prints
            if world > 1:
                raise  # every rank must take the same collective steps
            batch_line = {"error": f"{type(exc).__name__}: {exc}"[:400]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        t_cpu, cores = cpu_baseline(prob, steps=1)
        cpu = {"value": prob.m / t_cpu[0], "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "one full n=4096 solve (C++ restatement of the reference, OpenMP + "
                         "OpenBLAS LAPACK/BLAS), same workload"}

    # H = T^T I for 1, 8, 16 and 64 stacks with T resident (imcom_b200/t_reuse.py)
    # through each kernel, and the lookup tables' inverse FFT, own vs cuFFT
    # (imcom_b200/table_fft.py)
    t_reuse = table_fft = kappa_features = None
    if rank == 0 and world == 1 and not args.no_t_reuse:
        t_reuse = {k: child_measure("imcom_b200.t_reuse", "--kernel", k) for k in ("gemm", "stream")}
    if rank == 0 and world == 1 and not args.no_table_fft:
        table_fft = child_measure("imcom_b200.table_fft")
        # learned-kappa features: per-pixel scan vs neighbour table + band segments
        kappa_features = child_measure("imcom_b200.stages", "n4096", "--split",
                                       "--compare-features")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_DESC,
                       "n": n, "m": m, "nps": prob.nps, "lookup_side": 3 * prob.nps,
                       "eigensolver": args.eigensolver, "kappa": args.kappa,
                       "P_T_precision": ("split int8 digits on tcgen05 (7/6 slices), audited, "
                                         "FP64 fallback") if split else "fp64 (DMMA)",
                       "parallelism": f"replicas x{world}",
                       "l2": "flushed between timed steps (252 MB write)"},
            "plain_fp64_value": plain_value,
            "speedup_vs_plain_fp64": value / plain_value,
            "cached_stage": cached,
            "strict_target": strict,
            "stages_ms": avg,
            "stages_ms_plain": {k: statistics.mean(d[k] for d in plain_st) for k in plain_st[0]},
            "accuracy_vs_plain_fp64": accuracy,
            "kappa": kappa_info,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": t_e2e,
                    "ms_steps": [round(x, 3) for x in e2e_ms]},
            "gpu_launches": launches,
            "roofline": roof,
            "split_roofline": split_roof,
            "cpu_baseline": cpu,
            "batch": batch_line,
            "t_reuse": t_reuse,
            "table_fft": table_fft,
            "kappa_features": kappa_features,
            "clocks": ck,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    # a crash in native code prints the Python stack of every thread to stderr
    faulthandler.enable(all_threads=True)
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--eigensolver", choices=["dc", "library"], default="dc")
    ap.add_argument("--kappa", choices=["learned", "bisection"], default="learned")
    ap.add_argument("--precision", choices=["split", "fp64"], default="split",
                    help="P and T arithmetic of the fast path")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-patch measurement")
    ap.add_argument("--no-t-reuse", action="store_true",
                    help="skip the many-stack H = T^T I measurement")
    ap.add_argument("--no-table-fft", action="store_true",
                    help="skip the own-vs-cuFFT lookup-table FFT and the learned-kappa "
                         "features measurements")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
