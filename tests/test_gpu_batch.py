"""Ensembles of independent cases (sph_batch_*) on the GPU (needs a B200).

Stepping cases together on concurrent streams, with the host-controlled or
the device-controlled Krylov loop, must give exactly the results of stepping
each case alone (every kernel is deterministic), and the worker autotuner
must pick a valid worker count.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

pytestmark = pytest.mark.gpu

FIELDS = ("ux", "uy", "uz", "pres")


@pytest.mark.parametrize("threads", [32, 64])
def test_pair_pass_block_size_does_not_change_results(threads):
    P, p = decks.canyon(scale=0.12)
    out = []
    for t in (128, threads):
        sim = abi.Simulation(p, precision=layout.PREC_MIXED)
        sim.set_pair_block(t)
        sim.upload(P)
        for _ in range(2):
            sim.step(1)
        A, _, _ = sim.download()
        sim.close()
        out.append(A)
    for f in FIELDS:
        assert np.array_equal(out[0][f], out[1][f]), f


def _cases(refinement=0):
    out = []
    for k, (fn, n, re) in enumerate(((decks.cavity, 10, 400.0), (decks.tgv_box, 12, 1500.0),
                                     (decks.cavity, 14, 150.0))):
        P, p = fn(n=n, re=re, seed=100 + k)
        p.ppe_mode = layout.PPE_MIXED_IR
        p.ppe_tol = 1e-6
        p.ppe_coarse_block = 2
        p.ppe_refinement = refinement
        out.append((P, p))
    return out


@pytest.mark.parametrize("refinement", [0, 4], ids=["host_control", "device_control"])
def test_batch_equals_cases_stepped_alone(refinement):
    # device control (ppe_refinement 4) in the batch, host control alone:
    # the two give the same iterates
    cases = _cases(refinement)
    b = abi.Batch(cases, precision=layout.PREC_MIXED)
    b.set_workers(0)
    stats = b.step(4)     # under device control steps 2 and 3 replay a whole-step graph
    assert all(s.status == 0 and s.rel_residual <= 1e-6 for s in stats)
    for k, (P, p) in enumerate(cases):
        q = p.copy()
        q.ppe_refinement = 0
        sim = abi.Simulation(q, precision=layout.PREC_MIXED)
        sim.upload(P)
        for _ in range(4):
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
    w2, t, ms2 = b.autotune_shapes(probe_steps=1)
    assert 1 <= w2 <= len(cases) and t in (32, 64, 128) and ms2 > 0
    stats = b.step(1)
    assert all(s.status == 0 for s in stats)
    assert b.particles() == sum(len(P) for P, _ in cases)
    b.close()
