"""T applied to many image stacks: throughput of imcom_gpu_build_images.

The reference's production pattern builds T once (or reads it from the cache,
imcom_bisect.f90:47-62) and reuses it for every image stack observed with the
same dithers, mask and PSFs, forming H = T^T I per stack (imcom_build_image,
imcom_matrix.f90:754-790).  One stack is a matrix-vector product that streams
T (8 n m bytes) from HBM; S stacks at once are one FP64 GEMM (M = m, N = S,
K = n) that streams T once, so the work per stack falls until the GEMM turns
compute-bound near S = 4 x (FP64 peak / HBM bandwidth) ~ 20 stacks.  The
streaming kernel (IMCOM_OPT_STACK_KERNEL = 1) does the same sums with FP64
FMAs in passes of up to 8 stacks, without the GEMM's 128-wide stack tile.

    python -m imcom_b200.t_reuse [--n 4096 --m 4096 --stacks 1 8 16 64]
                                 [--kernel gemm|stream]

prints one JSON line: per stack count the device time of the chosen kernel
(T resident, L2 flushed before each launch, CUDA events on the library stream),
its HBM and FP64 rooflines, the same work as one per-stack launch per stack,
the end-to-end rate through the host-array entry point (stack copies in and
H copies out included), and the largest error against numpy's T^T I as a
fraction of the n-term dot-product error bound.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from .api import EPS, OPT_STACK_KERNEL, STACKS_GEMM, STACKS_STREAM, Solver

L2_BYTES = 126 * 1024 * 1024
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback 6.65 TB/s"


def _dgemm_peak(torch, dev):
    """cuBLAS FP64 GEMM TFLOP/s (torch.matmul, 8192^3, best of 3)."""
    n = 8192
    a = torch.randn((n, n), dtype=torch.float64, device=dev)
    b = torch.randn((n, n), dtype=torch.float64, device=dev)
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


def measure(n=4096, m=4096, stacks=(1, 8, 16, 64), reps=5, warmup=3, device=0, seed=0,
            kernel="gemm"):
    """kernel: "gemm" (the FP64 GEMM) or "stream" (the streaming kernel of
    up to 8 stacks per pass over T)."""
    import torch

    dev = torch.device("cuda", device)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(seed)
    hbm, hbm_src = _hbm_peak()
    f64 = _dgemm_peak(torch, dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    out = {"kernel": kernel,
           "workload": f"T resident ({n} inputs x {m} outputs, {8 * n * m / 1e6:.0f} MB), "
                       "H = T^T I for S stacks at once",
           "n": n, "m": m, "hbm_peak_gbs": hbm, "hbm_peak_source": hbm_src,
           "fp64_peak_tflops": f64, "fp64_peak_source": "cuBLAS DGEMM 8192^3 in this run",
           "l2": "flushed before every timed launch (252 MB write)", "runs": []}
    with Solver(device) as s:
        s.set_option(OPT_STACK_KERNEL, STACKS_STREAM if kernel == "stream" else STACKS_GEMM)
        # the geometry only fixes n and m; T's values do not change the work
        s.set_inputs(rng.uniform(0, 64, n), rng.uniform(0, 64, n), np.ones(n, dtype=np.int32),
                     rng.uniform(0, 64, m), rng.uniform(0, 64, m), I_i=rng.standard_normal(n))
        T = np.asfortranarray(rng.standard_normal((n, m)))
        s.load_T(T)
        stream = torch.cuda.ExternalStream(s.stream(), device=dev)

        def timed(fn):
            for _ in range(warmup):
                fn()
            ts = []
            for _ in range(reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                    e0.record(stream)
                    fn()
                    e1.record(stream)
                stream.synchronize()
                ts.append(e0.elapsed_time(e1) * 1e-3)
            return float(np.median(ts))

        t_one = timed(lambda: s.build_image(out=False))  # image_s_kernel, one stack
        out["per_stack_kernel_us"] = t_one * 1e6
        absT = np.abs(T)
        for S in stacks:
            I = rng.standard_normal((n, S)) + 1.0
            dI = torch.from_numpy(np.ascontiguousarray(I.T)).to(dev)
            dH = torch.empty((S, m), dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            t = timed(lambda: s.build_images_device(dI, dH))
            H = dH.cpu().numpy().T
            err = np.abs(H - T.T @ I) / (n * EPS * (absT.T @ np.abs(I)) + 1e-300)
            byts = 8.0 * (n * m + n * S + m * S)
            flops = 2.0 * n * m * S
            # end to end: host stacks in, host H out, through the host-array entry point
            Ih = np.asfortranarray(I)
            s.build_images(Ih)
            t0 = time.perf_counter()
            for _ in range(reps):
                s.build_images(Ih)
            t_e2e = (time.perf_counter() - t0) / reps
            out["runs"].append({
                "stacks": S, "us": t * 1e6, "stacks_per_s": S / t,
                "output_pixels_per_s": S * m / t,
                "speedup_vs_per_stack_launches": t_one * S / t,
                "hbm": {"algorithmic_bytes": byts, "achieved_gbs": byts / t / 1e9,
                        "frac": byts / t / 1e9 / hbm},
                "fp64": {"flops": flops, "achieved_tflops": flops / t / 1e12,
                         "frac": flops / t / 1e12 / f64},
                "e2e": {"stacks_per_s": S / t_e2e, "h2d_bytes": 8 * n * S, "d2h_bytes": 8 * m * S},
                "max_error_over_bound": float(err.max()),
            })
    return out


def main():
    ap = argparse.ArgumentParser(description="H = T^T I for many image stacks (T reuse)")
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--m", type=int, default=4096)
    ap.add_argument("--stacks", type=int, nargs="+", default=[1, 8, 16, 64])
    ap.add_argument("--kernel", choices=["gemm", "stream"], default="gemm")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args()
    print(json.dumps(measure(args.n, args.m, tuple(args.stacks), args.reps, device=args.device,
                             kernel=args.kernel)), flush=True)


if __name__ == "__main__":
    main()
