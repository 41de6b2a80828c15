"""Learned-kappa bracket: training data, GPU training and the weight format.

Training pairs come from the plain bisection (the reference's algorithm) on
seeded synthetic workloads: per output pixel the 12 features of
``imcom_gpu_kappa_features`` and the target log10(kappa).  Training runs on
the GPU through ``imcom_gpu_mlp_train`` (the project's own bf16 forward and
backward kernels, Adam in fp32).  The target normalisation is folded into the
last layer so the device MLP emits log10(kappa) and the log bracket
half-width in decades directly.

CLI: ``python -m imcom_b200.kappa_model [--seeds 49] [--out PATH]`` trains on
the n=4096 workload and writes the weights (npz).
"""
from __future__ import annotations

import argparse
import os

import numpy as np

NF, NH, NO = 12, 64, 2
NPARAM = NH * NF + NH + NH * NH + NH + NO * NH + NO
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                               "kappa_mlp_n4096.npz")


def unpack(p):
    p = np.asarray(p, dtype=np.float32)
    o = 0
    out = []
    for shape in ((NH, NF), (NH,), (NH, NH), (NH,), (NO, NH), (NO,)):
        size = int(np.prod(shape))
        out.append(p[o:o + size].reshape(shape))
        o += size
    return out


def pack(W1, b1, W2, b2, W3, b3):
    return np.concatenate([np.ravel(x).astype(np.float32) for x in (W1, b1, W2, b2, W3, b3)])


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    W1 = rng.standard_normal((NH, NF)) * np.sqrt(2.0 / NF)
    W2 = rng.standard_normal((NH, NH)) * np.sqrt(2.0 / NH)
    W3 = rng.standard_normal((NO, NH)) * np.sqrt(1.0 / NH)
    return pack(W1, np.zeros(NH), W2, np.zeros(NH), W3, np.zeros(NO))


def collect(solver, problems, targets, tol_rel=1e-3, maxnits=53):
    """Plain bisection on each (problem, U target); returns features (12, N)
    and log10 kappa (N)."""
    from .api import EPS
    feats, ys = [], []
    for prob, us in zip(problems, targets):
        solver.set_problem(prob)
        C = solver.psf_spectra()
        solver.build_A(out=False)
        solver.eigen_A(out=False)
        solver.build_B(out=False)
        solver.build_P(out=False)
        K, _, _ = solver.bisect_kappa(True, us, C * EPS, C / EPS, us * tol_rel, maxnits, C)
        feats.append(solver.kappa_features(True, us, C))
        ys.append(np.log10(K))
    return np.concatenate(feats, axis=1), np.concatenate(ys)


class KappaModel:
    """Trained weights plus the normalisation the device MLP expects."""

    def __init__(self, params, fmean, fstd, ymean, ystd):
        self.params = np.asarray(params, dtype=np.float32)
        self.fmean = np.asarray(fmean, dtype=np.float32)
        self.fstd = np.asarray(fstd, dtype=np.float32)
        self.ymean = float(ymean)
        self.ystd = float(ystd)

    def device_weights(self):
        """Weights with the target normalisation folded into the last layer."""
        W1, b1, W2, b2, W3, b3 = unpack(self.params)
        W3 = W3.copy()
        b3 = b3.copy()
        W3[0] *= self.ystd
        b3[0] = b3[0] * self.ystd + self.ymean
        b3[1] = b3[1] + np.log(self.ystd)
        return W1, b1, W2, b2, W3, b3, self.fmean, self.fstd

    def install(self, solver):
        solver.mlp_set_weights(*self.device_weights())

    def save(self, path):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.params, fmean=self.fmean, fstd=self.fstd, ymean=self.ymean,
                 ystd=self.ystd)

    @classmethod
    def load(cls, path):
        d = np.load(path)
        return cls(d["params"], d["fmean"], d["fstd"], float(d["ymean"]), float(d["ystd"]))


def train(solver, feat, y, epochs=40, batch=512, lr=2e-3, seed=1):
    fmean = feat.mean(axis=1)
    fstd = feat.std(axis=1)
    fstd[fstd < 1e-6] = 1.0
    ymean, ystd = float(y.mean()), float(max(y.std(), 1e-6))
    fn = (feat - fmean[:, None]) / fstd[:, None]
    yn = (y - ymean) / ystd
    p, loss = solver.mlp_train(fn, yn, init_params(seed), epochs=epochs, batch=batch, lr=lr,
                               seed=seed)
    return KappaModel(p, fmean, fstd, ymean, ystd), loss


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=49)
    ap.add_argument("--workload", default="n4096")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    args = ap.parse_args()
    from . import Solver, synth
    rng = np.random.default_rng(12345)
    probs = [synth.make(args.workload, seed=1000 + s) for s in range(args.seeds)]
    targets = list(10.0 ** rng.uniform(np.log10(3e-3), np.log10(3e-2), args.seeds))
    with Solver(0) as s:
        feat, y = collect(s, probs, targets)
        model, loss = train(s, feat, y, epochs=args.epochs)
    model.save(args.out)
    print(f"trained on {y.size} pixels from {args.seeds} seeds; loss {loss[0]:.4f} -> {loss[-1]:.4f}")


if __name__ == "__main__":
    main()
