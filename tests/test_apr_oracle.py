"""The CPU restatement of the APR pass (oracle/apr.py) against the
reference's own APR kernels compiled for the host (oracle/ref_apr_shim.cpp):
KERNEL_APR_condition3D_cell + Cell_index on a splitting state and on a
merging state (marks and cell numbers equal), KERNEL_cell_APR_3D on the
splitting state (the same records; positions within the cube-root rounding
of two libms).  The merge itself has no counterpart the reference runs: its
restatement is checked for mass and volume conservation and for putting the
merged record at the family's centre."""
import numpy as np
import pytest

from sph_b200 import decks, layout

import apr as apr_oracle
import refhost
import restated

needs_ref = pytest.mark.skipif(not refhost.apr_available(), reason="reference APR host build absent")


def _deck():
    P, p = decks.canyon(scale=0.12)
    P, p = decks.with_headroom(P, p, 1.0)   # room for every split the reference makes (it checks none)
    p.apr_max_level = 1
    p.apr_zone = 0.03
    p.seti("h_change", 1)
    return P, p


def _sorted_state(P, p):
    O = restated.Restated(P, p, 0)
    O.nnps()
    A, _, _ = O.download()
    g_idx, p_idx, g_str, g_end = O.export_nnps()
    return A, g_idx, p_idx, g_str, g_end


def _split_state():
    P, p = _deck()
    A, g_idx, _, g_str, g_end = _sorted_state(P, p)
    target = apr_oracle.zone_target(A, g_idx, p)
    family = np.arange(1, len(A) + 1, dtype=np.int32)
    return A, p, g_idx, g_str, g_end, target, family


@needs_ref
def test_condition_and_split_equal_reference_kernels():
    A, p, g_idx, g_str, g_end, target, family = _split_state()
    nc = p.geti("num_cells")
    first_free = int(g_str[nc])
    cond, flag = apr_oracle.condition(A, g_str, g_end, p, target, family)
    num, pos, neg = apr_oracle.numbering(flag)
    assert pos > 0 and neg == 0
    rcond, rcell, R, RM, RB = refhost.ref_apr_pass(A, g_str, g_end, p, target, family, first_free)
    assert np.array_equal(cond, rcond)
    assert np.array_equal(num, rcell)
    Q, T, F, ns, nm = apr_oracle.execute(A, g_str, g_end, p, target, family, cond, num, first_free)
    assert ns == pos and nm == 0
    for f in ("i_type", "p_type", "buffer_type", "m", "vol", "h", "h_ref", "m_ref", "ux", "uy", "uz", "pres", "rho"):
        assert np.array_equal(Q[f], R[f]), f
    for f in ("x", "y", "z"):
        assert np.allclose(Q[f], R[f], rtol=0, atol=2e-7), f
    assert np.array_equal(F, RB)
    assert np.array_equal(T, RM)
    # children from 8 records past the first free one (k_num_part + num_buffer + 8 * 1)
    assert Q["i_type"][first_free + 8] < 3 and np.all(Q["i_type"][first_free:first_free + 8] == 3)


def _merge_state():
    """The split state advanced by one pass, sorted again, with the target
    level dropped to 0: every family of children asks to merge."""
    A, p, g_idx, g_str, g_end, target, family = _split_state()
    nc = p.geti("num_cells")
    Q, T, F, ns, _, _ = apr_oracle.apr_pass(A, g_idx, g_str, g_end, p, family)
    assert ns > 0
    B, g2, p_idx, s2, e2 = _sorted_state(Q, p)
    F2 = F[p_idx]
    q = p.copy()
    q.apr_max_level = 0
    T2 = apr_oracle.zone_target(B, g2, q)
    return B, q, g2, s2, e2, T2, F2, ns


@needs_ref
def test_merge_marks_equal_reference_condition():
    B, q, g2, s2, e2, T2, F2, ns = _merge_state()
    nc = q.geti("num_cells")
    cond, flag = apr_oracle.condition(B, s2, e2, q, T2, F2)
    num, pos, neg = apr_oracle.numbering(flag)
    assert pos == 0 and neg > 0
    rcond, rcell, _, _, _ = refhost.ref_apr_pass(B, s2, e2, q, T2, F2, int(s2[nc]))
    assert np.array_equal(cond, rcond)
    assert np.array_equal(num, rcell)
    # at most one marked member per family of i_type 1 records (a cell marks
    # the family of its last candidate only, so some families wait for a
    # later pass); the search counts i_type 1 members only, so a candidate in
    # a buffer (i_type 2) marks itself
    marked = np.where(cond == -1)[0]
    inner = marked[B["i_type"][marked] == 1]
    assert 0 < len(inner) <= ns and len(set(F2[inner])) == len(inner)


def flag_count(B, s2, e2, q, T2, F2):
    """merging cells of a state: the tail records their numbers address"""
    _, flag = apr_oracle.condition(B, s2, e2, q, T2, F2)
    return int((flag < 0).sum())


def test_merge_conserves_mass_and_restores_the_parents():
    B, q, g2, s2, e2, T2, F2, ns = _merge_state()
    A, p, *_ = _split_state()
    live = lambda R: R["i_type"] < 3
    # families that can merge: eight active i_type 1 members
    fam, cnt = np.unique(F2[B["i_type"] == 1], return_counts=True)
    expected = int((cnt == 8).sum())
    assert expected > 0
    total = 0
    for _ in range(8):
        Q, T, F, nsplit, asked, nm = apr_oracle.apr_pass(B, g2, s2, e2, q, F2)
        assert nsplit == 0
        for f in ("m", "vol"):
            assert abs(Q[f][live(Q)].astype(np.float64).sum() - B[f][live(B)].astype(np.float64).sum()) <= \
                1e-6 * B[f][live(B)].astype(np.float64).sum(), f
        assert int(live(Q).sum()) == int(live(B).sum()) - 7 * nm
        # this pass's merged records (free records at the tail that became
        # active) sit where their parents were, with the parents' mass and h
        merged = np.where((B["i_type"] == 3) & (Q["i_type"] == 1))[0]
        assert len(merged) == nm and np.all(merged >= len(Q) - int((flag_count(B, s2, e2, q, T2, F2))))
        par = A[F[merged] - 1]            # family = the parent's index + 1 in the first sorted state
        for f in ("x", "y", "z"):
            assert np.allclose(Q[f][merged], par[f], rtol=0, atol=2e-7), f
        assert np.allclose(Q["m"][merged], par["m"], rtol=1e-6)
        assert np.allclose(Q["h"][merged], par["h"], rtol=1e-6)
        total += nm
        if nm == 0:
            break
        B, g2, p_idx, s2, e2 = _sorted_state(Q, q)
        F2 = F[p_idx]
    assert total == expected              # every family of inner records merged back
