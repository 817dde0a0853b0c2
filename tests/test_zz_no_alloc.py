"""The cell sort without device allocation, sph_nnps_sort_noalloc.

Callers that cannot call cudaMalloc (a host code that gives all of its device
memory to its own pool or arena, or one whose time loop must not allocate)
use this entry point to bin and sort particles with working memory that the
library holds in a static device array.  Its g_idx, p_idx, g_str and g_end
must equal those of the context path (sph_nnps + sph_nnps_export)
bit for bit, on calls in a row: the first deck sends a crowded cell through
the long-segment sort, the later ones have no long cells, so counters or
flags left over from an earlier call would show.  The file is
named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from sph_b200 import abi, decks, layout

SPH_ERR_BAD_ARG = -1
SPH_ERR_UNSUPPORTED = -7
SPH_NOALLOC_MAX_PARTICLES = 262144


def _context_sort(P, p):
    sim = abi.Simulation(p, precision=layout.PREC_MIXED)
    sim.upload(P)
    sim.nnps()
    out = sim.export_nnps()
    sim.close()
    return out


def _noalloc_sort(P, p):
    import torch
    dev = torch.device("cuda", 0)
    n = len(P)
    nc = p.geti("num_cells")
    cols = [torch.from_numpy(np.ascontiguousarray(P[f], dtype=np.float32)).to(dev) for f in ("x", "y", "z")]
    i_type = torch.from_numpy(np.ascontiguousarray(P["i_type"], dtype=np.int32)).to(dev)
    # outputs start as garbage so that an entry the call skips shows up
    g_idx = torch.full((n,), -7, dtype=torch.int32, device=dev)
    p_idx = torch.full((n,), -7, dtype=torch.int32, device=dev)
    g_str = torch.full((nc + 1,), -7, dtype=torch.int32, device=dev)
    g_end = torch.full((nc + 1,), -7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    st = abi.lib().sph_nnps_sort_noalloc(ctypes.byref(p), ptr(cols[0]), ptr(cols[1]), ptr(cols[2]), ptr(i_type), n,
                                         ptr(g_idx), ptr(p_idx), ptr(g_str), ptr(g_end), ctypes.c_void_p(stream))
    assert st == 0, abi.lib().sph_last_error().decode()
    torch.cuda.synchronize(dev)
    return [t.cpu().numpy() for t in (g_idx, p_idx, g_str, g_end)]


def _with_dummies(P, frac, seed):
    P = P.copy()
    rng = np.random.default_rng(seed)
    P["i_type"][rng.random(len(P)) < frac] = 3
    return P


def _crowded(P, count, seed):
    """`count` fluid particles moved onto the position of one other fluid
    particle, so that one cell holds them all."""
    P = P.copy()
    rng = np.random.default_rng(seed)
    fl = np.where((P["p_type"] == 1) & (P["i_type"] == 1))[0][:-1]
    c = fl[len(fl) // 2]
    pick = rng.permutation(fl[fl != c])[:count]
    for a in ("x", "y", "z"):
        P[a][pick] = P[a][c]
    return P


@pytest.mark.gpu
def test_noalloc_sort_equals_context_sort_on_two_calls():
    # first a deck whose crowded cell goes through the long-segment sort,
    # duplicated positions and scattered dummies; then decks without long
    # cells, so that a long-cell count or list left over would show
    P0, p0 = decks.nnps_stress()
    P1, p1 = decks.canyon(scale=0.3)                 # 62k particles, 13.5k cells
    P2, p2 = decks.caseh_mini()                      # 8k particles, 22k cells
    P2 = _with_dummies(P2, 0.03, seed=5)
    for P, p in ((P0, p0), (P1, p1), (P2, p2)):
        got = _noalloc_sort(P, p)
        ref = _context_sort(P, p)
        for name, a, b in zip(("g_idx", "p_idx", "g_str", "g_end"), got, ref):
            assert np.array_equal(a, b), name


@pytest.mark.gpu
def test_noalloc_sort_recovers_after_an_overfull_cell():
    # a cell of 5000 particles is beyond the 4096 the long-segment sort
    # holds: the call reports SPH_ERR_UNSUPPORTED; the flag it leaves in the
    # shared array must not fail the next call
    import torch
    P, p = decks.canyon(scale=0.3)
    Pc = _crowded(P, 5000, seed=11)
    dev = torch.device("cuda", 0)
    n, nc = len(Pc), p.geti("num_cells")
    cols = [torch.from_numpy(np.ascontiguousarray(Pc[f], dtype=np.float32)).to(dev) for f in ("x", "y", "z")]
    i_type = torch.from_numpy(np.ascontiguousarray(Pc["i_type"], dtype=np.int32)).to(dev)
    outs = [torch.empty(k, dtype=torch.int32, device=dev) for k in (n, n, nc + 1, nc + 1)]
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    st = abi.lib().sph_nnps_sort_noalloc(ctypes.byref(p), *[ptr(t) for t in cols], ptr(i_type), n,
                                         *[ptr(t) for t in outs],
                                         ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    assert st == SPH_ERR_UNSUPPORTED, st
    assert "4096" in abi.lib().sph_last_error().decode()
    got = _noalloc_sort(P, p)
    ref = _context_sort(P, p)
    for name, a, b in zip(("g_idx", "p_idx", "g_str", "g_end"), got, ref):
        assert np.array_equal(a, b), name


def test_noalloc_sort_rejects_more_particles_than_its_limit():
    # returns before any device work: runs without a GPU
    P, p = decks.caseh_mini()
    st = abi.lib().sph_nnps_sort_noalloc(ctypes.byref(p), None, None, None, None, SPH_NOALLOC_MAX_PARTICLES + 1,
                                         None, None, None, None, None)
    assert st == SPH_ERR_BAD_ARG
    assert "SPH_NOALLOC_MAX_PARTICLES" in abi.lib().sph_last_error().decode()
