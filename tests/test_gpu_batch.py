"""Ensembles of independent cases (sph_batch_*) on the GPU (needs a B200).

Stepping cases together on concurrent streams must give exactly the results
of stepping each case alone (every kernel is deterministic), and the worker
autotuner must pick a valid worker count.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

pytestmark = pytest.mark.gpu

FIELDS = ("ux", "uy", "uz", "pres")


def _cases():
    out = []
    for k, (fn, n, re) in enumerate(((decks.cavity, 10, 400.0), (decks.tgv_box, 12, 1500.0),
                                     (decks.cavity, 14, 150.0))):
        P, p = fn(n=n, re=re, seed=100 + k)
        p.ppe_mode = layout.PPE_MIXED_IR
        p.ppe_tol = 1e-6
        p.ppe_coarse_block = 2
        out.append((P, p))
    return out


def test_batch_equals_cases_stepped_alone():
    cases = _cases()
    b = abi.Batch(cases, precision=layout.PREC_MIXED)
    b.set_workers(0)
    stats = b.step(3)
    assert all(s.status == 0 and s.rel_residual <= 1e-6 for s in stats)
    for k, (P, p) in enumerate(cases):
        sim = abi.Simulation(p, precision=layout.PREC_MIXED)
        sim.upload(P)
        for _ in range(3):
            sim.step(1)
        A, _, _ = sim.download()
        sim.close()
        B = b.download(k)
        for f in FIELDS:
            assert np.array_equal(A[f], B[f]), (k, f)
    b.close()


def test_batch_autotune_picks_a_worker_count():
    cases = _cases()
    b = abi.Batch(cases, precision=layout.PREC_MIXED)
    w, ms = b.autotune(probe_steps=1)
    assert 1 <= w <= len(cases) and ms > 0
    stats = b.step(1)
    assert all(s.status == 0 for s in stats)
    assert b.particles() == sum(len(P) for P, _ in cases)
    b.close()
