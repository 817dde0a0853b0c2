"""Seeded synthetic decks (host logic, no GPU)."""
import numpy as np

from sph_b200 import decks


def test_ensemble_is_seeded_and_within_its_ranges():
    a = decks.ensemble(6, nmin=2000, nmax=6000)
    b = decks.ensemble(6, nmin=2000, nmax=6000)
    for (Pa, pa, ma), (Pb, pb, mb) in zip(a, b):
        assert ma == mb
        assert np.array_equal(Pa, Pb)
        assert 100.0 <= ma["re"] <= 2000.0
        assert 2000 <= ma["target_fluid"] <= 6000
        assert ma["edge"] == int(round(ma["target_fluid"] ** (1 / 3)))
        fluid = int((Pa["p_type"] == 1).sum())
        assert fluid == ma["edge"] ** 3
    kinds = [m["kind"] for _, _, m in a]
    assert kinds == ["cavity", "taylor-green"] * 3


def test_cavity_lid_and_viscosity():
    P, p = decks.cavity(n=8, re=400.0)
    L = 8 * 0.01
    lid = P["p_type"] == 9
    assert lid.any() and np.all(P["z"][lid] > L)
    assert abs(p.visc_fluid - 1.225 * L / 400.0) < 1e-12
    assert not np.any(P["buffer_type"])        # closed box: no buffers


def test_tgv_box_initial_field_is_divergence_free_pattern():
    P, _ = decks.tgv_box(n=8)
    fl = P["p_type"] == 1
    assert np.all(P["uz"][fl] == 0)
    assert np.abs(P["ux"][fl]).max() <= 1.0 and np.abs(P["ux"][fl]).max() > 0.5


def test_enthalpy_tables_deck_is_served_by_its_tables():
    """Every record the projection reaches (i_type < 3, p_type < 1000) has a
    table of at least two entries for its |p_type|, h and T ascend in every
    table (the lookup's bracket search relies on it), and the deck's
    enthalpies meet inner segments and the extrapolated lower end."""
    from sph_b200 import layout
    P, p, t = decks.enthalpy_tables_mini()
    assert p.geti("prop_table") == 1 and p.enthalpy_eqn == 1
    reach = (P["i_type"] < 3) & (P["p_type"] < 1000)
    for slot in np.unique(np.abs(P["p_type"][reach])):
        assert slot < layout.TABLE_SLOTS and t.size[slot] >= 2, slot
    for k in range(t.n_tables):
        for c in ("T", "h"):
            col = t.column(c, k)
            assert np.all(np.diff(col) > 0), (k, c)
    h = P["enthalpy"][reach & (np.abs(P["p_type"]) == 0)]
    wall = t.column("h", 0)
    assert (h < wall[0]).any() and ((h > wall[0]) & (h < wall[-1])).any()
