#!/usr/bin/env python
"""Benchmark: output pixels/s of the IMCOM solve path at n=4096.

A step is one full solve of the n=4096 workload (4 exposures of 32x32 input
pixels with U[-5,5] deg rotations and uniform dithers, Airy lambda/D = 0.5 px
(x) pixel PSFs, Gamma Gaussian sigma = 0.9 px, 64x64 output at 0.5 px,
lookup side 1728): PSF spectra -> A tables + assembly -> eigendecomposition
-> B tables + assembly -> P -> per-pixel kappa bisection (U < 1e-2, tolerance
1e-5) -> T -> S and H.  Synthetic seeded inputs (synth.make("n4096")).

  value  pixels/s with the inputs resident in HBM (no host copies timed),
         CUDA events on the library's stream, L2 flushed between steps.
  e2e    the same metric through the C-ABI with pinned host buffers: inputs
         copied in and H, K, U, S and T copied out inside every step.

``--impl reference`` times the CPU oracle (the reference's algorithm restated
in C++ with OpenMP + LAPACK/BLAS) on the same workload, all host cores.
Multi-GPU (``torchrun``): replicas only -- every rank solves its own
independent patch (seed = rank); value = all ranks' pixels / max rank time.
"""
from __future__ import annotations

import argparse
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
METRIC = "output pixels/s at n=4096 (learned-κ+mixed vs plain FP64 GPU, same U/Σ tol)"
UNIT = "pixels/s"
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


def fp64_gemm_peak(torch, dev):
    """cuBLAS DGEMM throughput (TFLOP/s) measured here: the FP64 roofline
    denominator (MEASURED_PEAKS.json carries HBM and bf16 only)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
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
        "config": {"workload": "n4096: 4x32x32 inputs (n=4096), 64x64 output (m=4096), "
                               "U mode U<1e-2 tol 1e-5, maxnits 53", "n": prob.n, "m": prob.m,
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
    nev_acc = {"plain": [], "learned": []}

    def device_step(use_learned):
        C = s.psf_spectra()
        kmin, kmax = C * 1.1102230246251565e-16, C / 1.1102230246251565e-16
        s.build_A(out=False)
        s.eigen_A(out=False)
        s.build_B(out=False)
        s.build_P(out=False)
        if use_learned:
            s.bisect_kappa_learned(UNOTS, US_MAX, kmin, kmax, US_TOL, MAXNITS, C, out=False)
        else:
            s.bisect_kappa(UNOTS, US_MAX, kmin, kmax, US_TOL, MAXNITS, C, out=False)
        s.build_T(out=False)
        s.build_S(out=False)
        s.build_image(out=False)

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

    def timed_steps(use_learned, nsteps):
        for _ in range(args.warmup):
            device_step(use_learned)
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
            device_step(use_learned)
            e1.record(stream)
            s.synchronize()
            sm.append(e0.elapsed_time(e1))
            st.append(s.stage_times())
        return sm, st, (s.launch_count() - l0) // max(1, nsteps)

    plain_ms, plain_st, _ = timed_steps(False, args.steps) if learned else (None, None, None)
    clocks = Clocks(local)
    clocks.start()
    step_ms, stage_ms, launches = timed_steps(learned, args.steps)
    torch.cuda.synchronize()
    ck = clocks.stop()
    barrier()
    t_step = max_over_ranks(statistics.mean(step_ms))
    value = world * prob.m / (t_step * 1e-3)
    # evaluation counts of the two kappa solvers on this workload (untimed)
    C = s.psf_spectra()
    _, _, nev_plain = s.bisect_kappa(UNOTS, US_MAX, C * 1.1102230246251565e-16,
                                     C / 1.1102230246251565e-16, US_TOL, MAXNITS, C)
    kappa_info = {"solver": "learned bracket + bisection replay" if learned else "bisection",
                  "mean_evaluations_plain": float(np.mean(nev_plain))}
    if learned:
        K0 = s.bisect_kappa(UNOTS, US_MAX, C * 1.1102230246251565e-16, C / 1.1102230246251565e-16,
                            US_TOL, MAXNITS, C)[0]
        K1, _, nev_l, fb = s.bisect_kappa_learned(UNOTS, US_MAX, C * 1.1102230246251565e-16,
                                                  C / 1.1102230246251565e-16, US_TOL, MAXNITS, C)
        t_plain = max_over_ranks(statistics.mean(plain_ms))
        kappa_info.update({
            "mean_evaluations_learned": float(np.mean(nev_l)),
            "no_bound_fraction": float(np.mean(fb)),
            "kappa_bit_identical_to_plain": bool(np.array_equal(K0, K1)),
            "model": model_src,
            "plain_fp64_value": world * prob.m / (t_plain * 1e-3),
            "bisect_ms_plain": statistics.mean(d["bisect"] for d in plain_st),
            "bisect_ms_learned": statistics.mean(d["bisect"] for d in stage_ms),
        })

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
        C = s.psf_spectra()
        kmin, kmax = C * 1.1102230246251565e-16, C / 1.1102230246251565e-16
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

    # ---- roofline of the dominant own kernel -------------------------------
    avg = {k: statistics.mean(d[k] for d in stage_ms) for k in stage_ms[0]}
    n, m = prob.n, prob.m
    peaks = measured_peaks()
    dgemm_peak = fp64_gemm_peak(torch, dev) if rank == 0 else None
    # per-stage algorithmic work: FP64 GEMM flops 2 n^2 m (P and T)
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
        roof = {"kernel": "trd_panel_kernel (eigen_A tridiagonalisation)", "bound": "hbm",
                "achieved": ach, "peak": pk, "unit": "GB/s", "frac": ach / pk,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                "algorithmic_bytes": byts, "traffic": None}
    elif dom in ("build_P", "build_T"):
        ach = 2.0 * n * n * m / (avg[dom] * 1e-3) / 1e12
        roof = {"kernel": dom, "bound": "tensor", "achieved": ach, "peak": dgemm_peak,
                "unit": "TFLOP/s", "frac": ach / dgemm_peak if dgemm_peak else None,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 DMMA path)",
                "traffic": None}
    else:
        # interpolation / others: HBM bytes written (A n^2 or B n m doubles) as the
        # algorithmic traffic; the kernel is bound by L1/L2 gathers of the tables
        byts = {"build_A": 8.0 * n * n, "build_B": 8.0 * n * m}.get(dom, 8.0 * n * m)
        ach = byts / (avg[dom] * 1e-3) / 1e9
        pk = peaks.get("hbm_gbs", 6650.0)
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": pk, "unit": "GB/s",
                "frac": ach / pk, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                "traffic": None}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        t_cpu, cores = cpu_baseline(prob, steps=1)
        cpu = {"value": prob.m / t_cpu[0], "unit": UNIT, "cores": cores, "kind": "port",
               "sample": "one full n=4096 solve (C++ restatement of the reference, OpenMP + "
                         "OpenBLAS LAPACK/BLAS), same workload"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "n4096: 4x32x32 inputs (n=4096), rotations U[-5,5] deg, Airy "
                                   "lambda/D=0.5 px PSF, 64x64 output at 0.5 px (m=4096), "
                                   "U mode U<1e-2 tol 1e-5, maxnits 53",
                       "n": n, "m": m, "nps": prob.nps, "lookup_side": 3 * prob.nps,
                       "eigensolver": args.eigensolver, "kappa": args.kappa,
                       "P_T_precision": "fp64 (DMMA)",
                       "parallelism": f"replicas x{world}",
                       "l2": "flushed between timed steps (252 MB write)"},
            "stages_ms": avg,
            "kappa": kappa_info,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": t_e2e},
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": ck,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--eigensolver", choices=["dc", "library"], default="dc")
    ap.add_argument("--kappa", choices=["learned", "bisection"], default="learned")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
