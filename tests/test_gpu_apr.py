"""Adaptive particle refinement (sph_apr) on the GPU (needs a B200).

One splitting pass against the CPU restatement (oracle/apr.py) on the same
sorted state: the same cells split, the same parents become dummies, the
children carry m/8, vol/8, h/2 and sit at the parent's position +-
cbrt(m/rho)/4 (within FP32 rounding of the cube root).  Mass is conserved
and the refined deck keeps stepping.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

import apr as apr_oracle

pytestmark = pytest.mark.gpu


def _deck():
    P, p = decks.canyon(scale=0.12)
    P, p = decks.with_headroom(P, p, 0.3)
    p.apr_max_level = 1
    p.apr_zone = 0.03
    p.seti("h_change", 1)
    p.ppe_mode = layout.PPE_MIXED_IR
    p.ppe_coarse_block = 2
    return P, p


def test_apr_split_matches_cpu_restatement():
    P, p = _deck()
    sim = abi.Simulation(p, precision=layout.PREC_MIXED)
    sim.upload(P)
    sim.nnps()
    A, _, _ = sim.download()
    _, _, g_str, g_end = sim.export_nnps()
    E, cells, wanted = apr_oracle.split(A, g_str, g_end, p)
    ns, nw = sim.apr()
    assert ns > 0 and (ns, nw) == (cells, wanted)
    B, _, _ = sim.download()
    for f in ("i_type", "p_type", "buffer_type", "m", "vol", "h", "ux", "pres"):
        assert np.array_equal(B[f], E[f]), f
    for f in ("x", "y", "z"):
        assert np.allclose(B[f], E[f], rtol=0, atol=1e-6), f
    live = lambda R: R["m"][R["i_type"] < 3].astype(np.float64).sum()
    assert abs(live(B) - live(A)) <= 1e-6 * live(A)
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
