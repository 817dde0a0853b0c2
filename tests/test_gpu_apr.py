"""Adaptive particle refinement (sph_apr) on the GPU (needs a B200).

Splitting and merging passes against the CPU restatement (oracle/apr.py,
itself checked against the reference's own APR kernels in
tests/test_apr_oracle.py) on the same sorted state: the same cells split,
the same families merge, the same records become dummies; children carry
m/8, vol/8, h/2 at the parent's position +- cbrt(m/rho)/4, merged records
the sums and means of their family (positions within FP32 cube-root
rounding).  Mass is conserved and the refined deck keeps stepping.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

import apr as apr_oracle

pytestmark = pytest.mark.gpu

EXACT = ("i_type", "p_type", "buffer_type", "m", "vol", "h", "h_ref", "m_ref", "ux", "uy", "uz", "pres")


def _deck():
    P, p = decks.canyon(scale=0.12)
    P, p = decks.with_headroom(P, p, 0.3)
    p.apr_max_level = 1
    p.apr_zone = 0.03
    p.seti("h_change", 1)
    p.ppe_mode = layout.PPE_MIXED_IR
    p.ppe_coarse_block = 2
    return P, p


def _state(sim):
    sim.nnps()
    A, _, _ = sim.download()
    g_idx, _, g_str, g_end = sim.export_nnps()
    fam, tgt, _ = sim.apr_state()
    return A, g_idx, g_str, g_end, fam


def _compare(B, E):
    for f in EXACT:
        assert np.array_equal(B[f], E[f]), f
    for f in ("x", "y", "z"):
        assert np.allclose(B[f], E[f], rtol=0, atol=2e-7), f


def test_apr_split_matches_cpu_restatement():
    P, p = _deck()
    sim = abi.Simulation(p, precision=layout.PREC_MIXED)
    sim.upload(P)
    A, g_idx, g_str, g_end, fam = _state(sim)
    assert not fam.any()                       # no family before the first pass
    E, T, F, cells, wanted, merged = apr_oracle.apr_pass(A, g_idx, g_str, g_end, p)
    ns, nw = sim.apr()
    assert ns > 0 and (ns, nw) == (cells, wanted) and merged == 0
    B, _, _ = sim.download()
    _compare(B, E)
    fam2, tgt2, nm = sim.apr_state()
    assert nm == 0
    assert np.array_equal(fam2, F) and np.array_equal(tgt2, T)
    live = lambda R: R["m"][R["i_type"] < 3].astype(np.float64).sum()
    assert abs(live(B) - live(A)) <= 1e-6 * live(A)
    sim.close()


def test_apr_merge_matches_cpu_restatement():
    P, p = _deck()
    sim = abi.Simulation(p, precision=layout.PREC_MIXED)
    sim.upload(P)
    for _ in range(8):                         # refine until no cell asks
        if sim.apr()[0] == 0:
            break
    q = p.copy()
    q.apr_max_level = 0                        # target level 0: the children's families merge
    sim.set_params(q)
    total = 0
    for _ in range(8):
        A, g_idx, g_str, g_end, fam = _state(sim)
        E, T, F, cells, wanted, merged = apr_oracle.apr_pass(A, g_idx, g_str, g_end, q, fam)
        ns, nw = sim.apr()
        _, _, nm = sim.apr_state()
        assert (ns, nm) == (0, merged)
        B, _, _ = sim.download()
        _compare(B, E)
        live = lambda R: R["m"][R["i_type"] < 3].astype(np.float64).sum()
        assert abs(live(B) - live(A)) <= 1e-6 * live(A)
        total += nm
        if nm == 0:
            break
    assert total > 0
    B, _, _ = sim.download()
    assert int((B["i_type"] < 3).sum()) <= int((P["i_type"] < 3).sum()) + 7 * 400
    sim.close()


def test_refined_deck_keeps_stepping():
    P, p = _deck()
    sim = abi.Simulation(p, precision=layout.PREC_MIXED)
    sim.upload(P)
    sim.step(1)
    ns, _ = sim.apr()
    assert ns > 0
    for _ in range(2):
        s = sim.step(1)
        assert s.status == 0 and s.rel_residual <= 1e-6
    B, _, _ = sim.download()
    assert int((B["i_type"] < 3).sum()) == int((P["i_type"] < 3).sum()) + 7 * ns
    for f in ("ux", "uy", "uz", "pres"):
        assert np.all(np.isfinite(B[f][B["i_type"] < 3])), f
    sim.close()
