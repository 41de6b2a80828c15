"""Batched patches: several contexts on one GPU, each on a share of the SMs,
solving independent patches of uneven size (masked input pixels).

* Every patch of a batch solved with three contexts side by side meets the
  bars a GPU solve meets against the oracle when compared with a
  one-context solve of that patch (kappa 1e-6 relative, U/S 1e-6 relative,
  H 1e-8 normwise).  The SM share changes grid shapes and so the rounding
  of the eigensolver's reductions, by the same amount as two runs of one
  context differ (~1e-9 relative in U at a 1e-6 leakage target on these
  patches).
* One patch of a batch against the oracle.
* Results come back in input order whatever order the queue deals them in.
* The autotuner returns the best of its candidate configurations (concurrency
  x tail cluster) and caches the choice.
* The tridiagonalisation tail in an 8-CTA cluster, and no cluster tail at
  all, agree with the default.
"""
import numpy as np
import pytest

from imcom_b200 import batch
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KW = dict(UnotS=True, US_max=1e-6, US_tol=1e-8, maxnits=53)


def relmax(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def check_close(g, r):
    assert np.max(np.abs(g.K / r.K - 1)) < 1e-6
    assert relmax(g.US, r.US) < 1e-6
    assert relmax(g.S, r.S) < 1e-6
    assert np.linalg.norm(g.H - r.H) <= 1e-8 * np.linalg.norm(r.H)


@pytest.fixture(scope="module")
def patches():
    return batch.make_batch(4, seed0=200)


@pytest.fixture(scope="module")
def batched(patches):
    with batch.BatchSolver(3) as b:
        assert b.share == batch.device_sms() // 3
        return b.solve(patches, **KW)


def test_batch_matches_single_context(solver, patches, batched):
    assert batched.concurrency == 3
    assert batched.pixels == sum(p.m for p in patches)
    assert len(batched.timeline) == len(patches)
    for p, g in zip(patches, batched.results):
        assert g.H.shape[0] == p.m  # results in input order
        r = solver.solve(p, keep=(), **KW)
        check_close(g, r)


def test_batch_patch_vs_oracle(patches, batched):
    i = int(np.argmin([p.n for p in patches]))
    r = O.solve(patches[i], **KW)
    g = batched.results[i]
    assert np.max(np.abs(g.K / r.K - 1)) < 1e-6
    assert relmax(g.US, r.US) < 1e-6
    assert np.linalg.norm(g.H - r.H) <= 1e-8 * np.linalg.norm(r.H)


def test_masked_inputs_are_uneven(patches):
    ns = [p.n for p in patches]
    assert len(set(ns)) == len(ns) and any(n % 4 for n in ns)


def test_autotune_picks_a_candidate(patches):
    sample = patches[:2]
    batch._TUNED.clear()
    tune = batch.autotune(sample, candidates=(1, 2), tails=(0, -1), **KW)
    assert tune.concurrency in (1, 2) and tune.tail_ctas in (0, -1)
    assert set(tune.rates) == {(1, 0), (1, -1), (2, 0), (2, -1)}
    assert tune.rates[(tune.concurrency, tune.tail_ctas)] == max(tune.rates.values())
    assert batch.autotune(sample, candidates=(1, 2), tails=(0, -1), **KW) is tune


def test_tail_cluster_settings_agree(solver, patches):
    """The cluster tail (16 or 8 CTAs) and the panel kernel to the end give
    the same solve to the oracle-level bars."""
    p = patches[0]
    r = solver.solve(p, keep=(), **KW)
    for t in (8, -1):
        with batch.BatchSolver(1, tail_ctas=t) as b:
            g = b.solve([p], **KW).results[0]
        check_close(g, r)
