"""Property tables (prop_table = 1) of the enthalpy form on the GPU, through
the C ABI (needs a B200).

* The step with the two-material tables (htoT of table |p_type|) against
  the oracle, which is bit-exact against the reference built with
  enthalpy_eqn 1 reading the same tables with its own read_table
  (tests/test_oracle.py): the same bars as the built-in-table enthalpy step.
* The step refuses to run without tables, with a slot the records need left
  empty or shorter than two entries, or with a record whose |p_type| no slot
  serves; sph_set_prop_tables refuses tables outside the 50 entries.  Every
  refusal is a host check made before any launch.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

import restated

pytestmark = pytest.mark.gpu

FP32_TOL = 2e-4
FP64_TOL = 2e-6   # the deck's MOST layer is FP32 in both forms
FIELDS = ["ux", "uy", "uz", "pres", "vis_t", "flt_s", "temp", "concn", "enthalpy"]


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / scale)


@pytest.mark.parametrize("precision,tol", [(layout.PREC_MIXED, FP32_TOL), (layout.PREC_FP64, FP64_TOL)],
                         ids=["fp32", "fp64"])
def test_table_step_matches_oracle(precision, tol):
    P, p, tables = decks.enthalpy_tables_mini()
    q = p.copy()
    q.ppe_mode = layout.PPE_REF_SWEEP
    sim = abi.Simulation(q, precision=precision)
    sim.set_prop_tables(tables)
    sim.upload(P)
    O = restated.Restated(P, q, precision)
    O.set_tables(tables)
    for _ in range(3):
        sim.step(1)
        O.step(1, mode=layout.PPE_REF_SWEEP)
    A, A2, A3 = sim.download()
    B, B2, B3 = O.download()
    sim.close()
    bad = {f: e for f, e in ((f, rel_err(A[f], B[f])) for f in FIELDS) if not e <= tol}
    assert not bad, bad
    assert rel_err(A2["enthalpy0"], B2["enthalpy0"]) <= max(tol, 4 * float(np.finfo(np.float32).eps))
    # the tables, not the corium table, set the temperature
    inner = (B["p_type"] == 1) & (B["buffer_type"] == 0)
    h0 = B2["enthalpy0"][inner].astype(np.float64)
    assert np.allclose(A["temp"][inner], np.interp(h0, decks.TABLE_FLUID["h"], decks.TABLE_FLUID["T"]), rtol=1e-4)


def _sim(P, p):
    q = p.copy()
    q.ppe_mode = layout.PPE_REF_SWEEP
    sim = abi.Simulation(q, precision=layout.PREC_MIXED)
    sim.upload(P)
    return sim


def test_step_without_tables_is_refused():
    P, p, _ = decks.enthalpy_tables_mini()
    sim = _sim(P, p)
    with pytest.raises(abi.SphError):
        sim.step(1)
    sim.close()


def test_step_with_a_needed_slot_too_short_is_refused():
    P, p, _ = decks.enthalpy_tables_mini()
    one = {c: v[:1] for c, v in decks.TABLE_WALL.items()}
    sim = _sim(P, p)
    sim.set_prop_tables(layout.PropTables.from_columns([one, decks.TABLE_FLUID]))
    with pytest.raises(abi.SphError):
        sim.step(1)
    # only the fluid slot: the walls' slot 0 is empty
    sim.set_prop_tables(layout.PropTables.from_columns([{c: [] for c in decks.TABLE_WALL}, decks.TABLE_FLUID]))
    with pytest.raises(abi.SphError):
        sim.step(1)
    # with both tables the same context steps
    _, _, tables = decks.enthalpy_tables_mini()
    sim.set_prop_tables(tables)
    sim.step(1)
    sim.close()


def test_step_with_an_unserved_p_type_is_refused():
    P, p, tables = decks.enthalpy_tables_mini()
    P = P.copy()
    k = int(np.nonzero((P["p_type"] == 0) & (P["i_type"] < 3))[0][0])
    P["p_type"][k] = 12
    sim = _sim(P, p)
    sim.set_prop_tables(tables)
    with pytest.raises(abi.SphError):
        sim.step(1)
    sim.close()


def test_tables_outside_the_entries_are_refused():
    P, p, tables = decks.enthalpy_tables_mini()
    sim = _sim(P, p)
    bad = layout.PropTables.from_buffer_copy(bytes(tables))
    bad.index[1], bad.size[1] = 45, 6
    with pytest.raises(abi.SphError):
        sim.set_prop_tables(bad)
    sim.close()


@pytest.mark.parametrize("precision", [layout.PREC_MIXED, layout.PREC_FP64], ids=["fp32", "fp64"])
@pytest.mark.parametrize("tables", [False, True], ids=["corium", "tables"])
def test_energy_conversions_match_oracle_bit_for_bit(precision, tables):
    """sph_energy_convert (KERNEL_clc_TemptoEnthalpy / KERNEL_clc_EnthalpytoTemp)
    against the oracle, which is bit-exact against the reference's kernels
    (tests/test_oracle.py): one interpolation per record, each step rounded
    as the reference's arithmetic rounds it, so the results are equal.
    Temperatures and enthalpies span every branch of the lookup; with the
    tables the deck's IBM markers (|p_type| 1000, no table) keep their
    values."""
    if tables:
        P, p, t = decks.enthalpy_tables_mini()
    else:
        (P, p), t = decks.enthalpy_mini(), None
    P = P.copy()
    rng = np.random.default_rng(9)
    P["temp"] = rng.uniform(200.0, 3000.0, len(P)).astype(np.float32)
    sim = abi.Simulation(p, precision=precision)
    O = restated.Restated(P, p, precision)
    if t is not None:
        sim.set_prop_tables(t)
        O.set_tables(t)
    sim.upload(P)
    sim.enthalpy_from_temperature()
    A, A2, _ = sim.download()
    O.temp_to_enthalpy()
    B, B2, _ = O.download()
    assert np.array_equal(A["enthalpy"], B["enthalpy"])
    assert np.array_equal(A2["enthalpy0"], B2["enthalpy0"])
    if t is not None:
        markers = P["p_type"] == 1000
        assert np.array_equal(A["enthalpy"][markers], P["enthalpy"][markers])
    Q = np.array(A, copy=True)
    Q["enthalpy"] = rng.uniform(-7.0e5, 1.5e6, len(Q)).astype(np.float32)
    sim.upload(Q)
    sim.temperature_from_enthalpy()
    C, _, _ = sim.download()
    O2 = restated.Restated(Q, p, precision)
    if t is not None:
        O2.set_tables(t)
    O2.enthalpy_to_temp()
    D, _, _ = O2.download()
    sim.close()
    assert np.array_equal(C["temp"], D["temp"])


def test_energy_conversion_needs_tables_when_asked_for():
    P, p, _ = decks.enthalpy_tables_mini()
    sim = _sim(P, p)
    with pytest.raises(abi.SphError):
        sim.enthalpy_from_temperature()
    sim.close()
