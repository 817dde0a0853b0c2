"""Parity at the benchmark decks' full sizes (needs a B200).

The small decks of test_gpu_parity.py pin every kernel; these tests check
that nothing changes at the sizes the benchmark runs: cell hash, sort
permutation, cell ranges and the canonical neighbour lists bit-exact against
the CPU oracle on

  * the urban canyon at full size (240 x 120 x 60 fluid lattice, 1.9 M records),
  * the 64^3 Taylor-Green box with its periodic ghost layers,
  * the uniform cube array at scale 0.5 (2.4 x 1.2 x 0.4 m, ~1.2 M records),
  * the cube array at scale 0.2 after the GPU's two-level APR passes,

and one step of the reference's own semantics (one PPE sweep) on the canyon
at scale 0.3 within the FP32 step bar of test_gpu_parity.py.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

import restated

pytestmark = pytest.mark.gpu

FP32_TOL = 2e-4
FIELDS = ["ux", "uy", "uz", "pres", "vis_t", "flt_s", "fbx", "fby", "fbz", "fmx", "fmy", "hmz"]


def _nnps_equal(P, p, boxes=None):
    sim = abi.Simulation(p, precision=layout.PREC_MIXED)
    if boxes is not None:
        sim.set_ib_boxes(boxes)
    sim.upload(P)
    sim.nnps()
    got = sim.export_nnps()
    off, lst = sim.neighbors()
    sim.close()
    O = restated.Restated(P, p, 0)
    O.nnps()
    ref = O.export_nnps()
    for name, a, b in zip(("g_idx", "p_idx", "g_str", "g_end"), got, ref):
        assert np.array_equal(a, b), name
    ooff, olst = O.neighbors()
    assert np.array_equal(off, ooff), "list offsets"
    assert np.array_equal(lst, olst), "list entries"
    return len(lst)


def test_nnps_bit_exact_full_canyon():
    P, p = decks.canyon(scale=1.0)
    assert len(P) > 1_800_000
    assert _nnps_equal(P, p) > 150_000_000


def test_nnps_bit_exact_tgv_64():
    P, p = decks.tgv_periodic(n=64)
    assert _nnps_equal(P, p) > 0


def test_nnps_bit_exact_uniform_cube_array_half_scale():
    P, p, boxes = decks.cube_array(scale=0.5)
    assert len(P) > 1_000_000
    assert _nnps_equal(P, p, boxes) > 0


def test_nnps_bit_exact_refined_cube_array():
    P, p, boxes = decks.cube_array(scale=0.2, apr=True)
    p.ppe_pair_h = 1
    sim = abi.Simulation(p, precision=layout.PREC_MIXED)
    sim.set_ib_boxes(boxes)
    sim.upload(P)
    split = 0
    for _ in range(16):
        ns, _ = sim.apr()
        split += ns
        if ns == 0:
            break
    R, _, _ = sim.download()
    sim.close()
    assert split > 0
    assert _nnps_equal(R, p, boxes) > 0


def test_reference_step_canyon_scale_03():
    P, p = decks.canyon(scale=0.3)
    q = p.copy()
    q.ppe_mode = layout.PPE_REF_SWEEP
    sim = abi.Simulation(q, precision=layout.PREC_MIXED)
    sim.upload(P)
    O = restated.Restated(P, q, 0)
    sim.step(1)
    O.step(1, mode=layout.PPE_REF_SWEEP)
    A, _, _ = sim.download()
    B, _, _ = O.download()
    sim.close()
    for f in FIELDS:
        a, b = A[f].astype(np.float64), B[f].astype(np.float64)
        err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)
        assert err <= FP32_TOL, (f, err)
