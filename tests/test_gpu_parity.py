"""CUDA path vs the CPU oracle, through the C ABI (needs a B200).

Bars:
  * NNPS (g_idx, p_idx, g_str, g_end) and the canonical neighbour lists are
    bit-exact against the oracle, which is itself bit-exact against the
    reference's own host build (tests/test_oracle.py);
  * one reference-compatible step (PPE as one Jacobi sweep): every P1 field
    within a relative error of FP32_TOL (FP32 form, FMA contraction and
    summation-order rounding) or FP64_TOL (FP64 form) of the oracle in the
    same precision, measured as max|a-b| / max|b| per field.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

import restated

pytestmark = pytest.mark.gpu

FP32_TOL = 2e-4
FP64_TOL = 1e-9
# MOST (functions_MOST.cuh:151-322) is evaluated in FP32 with float
# transcendentals in both forms, as in the reference; fields it drives carry
# FP32 rounding (logf/atanf of CUDA vs the host libm) even in the FP64 form.
MOST_FIELDS = {"fmx", "fmy", "hmz", "float1", "float2", "float3"}
FP64_MOST_TOL = 2e-6
FIELDS = ["ux", "uy", "uz", "pres", "vis_t", "flt_s", "fbx", "fby", "fbz", "fmx", "fmy", "hmz",
          "float1", "float2", "float3", "temp", "concentration", "k_turb", "e_turb"]


def stored_tol(arr, tol):
    """A field stored in FP32 (part2/part3 keep the reference's float layout)
    cannot agree closer than a few FP32 ulps, whatever precision computed it."""
    if np.asarray(arr).dtype == np.float32:
        return max(tol, 4 * float(np.finfo(np.float32).eps))
    return tol


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / scale)


def _decks():
    out = [("caseh_mini", decks.caseh_mini())]
    out.append(("caseh_ddf_monaghan", decks.caseh_mini(turbulence="DDF", viscous=layout.MONAGHAN, seed=7)))
    out.append(("canyon_small", decks.canyon(scale=0.12)))
    # the other kernel functions of functions_KNL.cuh and Euler time stepping
    for k in ("Gaussian", "Quintic", "Quartic", "Wendland2", "Wendland4"):
        out.append(("caseh_" + k.lower(), decks.caseh_mini(nx=12, ny=6, nz=5, kernel=k)))
    P, p = decks.caseh_mini(nx=12, ny=6, nz=5)
    p.seti("time_type", layout.EULER)
    out.append(("caseh_euler", (P, p)))
    # triply periodic box with periodic ghost records
    out.append(("tgv_periodic", decks.tgv_periodic(n=8)))
    # the pressure force's difference form (pressure_force_form 1)
    P, p = decks.canyon(scale=0.12)
    p.pressure_force_form = 1
    out.append(("canyon_difference_form", (P, p)))
    return out


DECKS = _decks()
NNPS_DECKS = DECKS + [("nnps_stress", decks.nnps_stress())]


@pytest.mark.parametrize("name,deck", NNPS_DECKS, ids=[d[0] for d in NNPS_DECKS])
def test_nnps_bit_exact(name, deck):
    P, p = deck
    sim = abi.Simulation(p, precision=layout.PREC_MIXED)
    sim.upload(P)
    sim.nnps()
    g_idx, p_idx, g_str, g_end = sim.export_nnps()
    O = restated.Restated(P, p, 0)
    O.nnps()
    og, op, os_, oe = O.export_nnps()
    assert np.array_equal(g_idx, og)
    assert np.array_equal(p_idx, op)
    assert np.array_equal(g_str, os_)
    occupied = os_ >= 0
    assert np.array_equal(g_end[occupied], oe[occupied])
    off, lst = sim.neighbors()
    ooff, olst = O.neighbors()
    assert np.array_equal(off, ooff)
    assert np.array_equal(lst, olst)
    sim.close()


def _run_pair(P, p, precision, nsteps, mode=layout.PPE_REF_SWEEP):
    q = p.copy()
    q.ppe_mode = mode
    sim = abi.Simulation(q, precision=precision)
    sim.upload(P)
    O = restated.Restated(P, q, precision)
    for _ in range(nsteps):
        sim.step(1)
        O.step(1, mode=mode)
    A, A2, A3 = sim.download()
    B, B2, B3 = O.download()
    sim.close()
    return A, A2, A3, B, B2, B3


@pytest.mark.parametrize("precision,tol", [(layout.PREC_MIXED, FP32_TOL), (layout.PREC_FP64, FP64_TOL)],
                         ids=["fp32", "fp64"])
@pytest.mark.parametrize("name,deck", DECKS, ids=[d[0] for d in DECKS])
def test_step_matches_oracle(name, deck, precision, tol):
    P, p = deck
    A, A2, A3, B, B2, B3 = _run_pair(P, p, precision, nsteps=3)
    has_most = bool((P["MOST_buffer"] == 1).any())
    errs = {f: rel_err(A[f], B[f]) for f in FIELDS}
    # with MOST particles the FP32 wall-layer forcing reaches every field
    # through the momentum balance; the MOST-free deck below checks FP64 tightly
    lim = {f: (FP64_MOST_TOL if (precision == layout.PREC_FP64 and has_most) else tol) for f in FIELDS}
    bad = {f: e for f, e in errs.items() if e > lim[f]}
    assert not bad, bad
    for f in ("ftotalx", "ftotaly", "ftotalz", "fpx", "fpy", "fpz", "inv_cm_xx", "inv_cm_xy", "inv_cm_zz"):
        assert rel_err(A3[f], B3[f]) <= stored_tol(B3[f], tol * 10), f
    for f in ("SR", "rho_ref", "ux0"):
        assert rel_err(A2[f], B2[f]) <= stored_tol(B2[f], tol * 10), f


def test_fp64_step_without_most_matches_oracle_tightly():
    P, p = decks.caseh_mini(seed=11)
    P["MOST_buffer"] = 0
    A, A2, A3, B, B2, B3 = _run_pair(P, p, layout.PREC_FP64, nsteps=3)
    errs = {f: rel_err(A[f], B[f]) for f in FIELDS}
    bad = {f: e for f, e in errs.items() if e > FP64_TOL}
    assert not bad, bad


THERMAL = {"all": (1, 1, 1), "conduction": (1, 0, 0), "boussinesq": (0, 1, 0), "concentration": (0, 0, 1)}


@pytest.mark.parametrize("precision,tol", [(layout.PREC_MIXED, FP32_TOL), (layout.PREC_FP64, FP64_TOL)],
                         ids=["fp32", "fp64"])
@pytest.mark.parametrize("name", list(THERMAL))
def test_thermal_step_matches_oracle(name, precision, tol):
    """Conduction, Boussinesq buoyancy and concentration transport: the
    oracle is bit-exact against the reference for these switches
    (tests/test_oracle.py); the CUDA path agrees with it to the step bar
    (the deck has MOST particles, whose FP32 forcing sets the FP64 bar)."""
    P, p = decks.thermal_mini(*THERMAL[name])
    A, A2, A3, B, B2, B3 = _run_pair(P, p, precision, nsteps=3)
    lim = FP64_MOST_TOL if precision == layout.PREC_FP64 else tol
    errs = {f: rel_err(A[f], B[f]) for f in FIELDS + ["concn"]}
    bad = {f: e for f, e in errs.items() if e > lim}
    assert not bad, bad
    for f in ("ftotalx", "ftotaly", "ftotalz", "dtemp", "dconcn"):
        assert rel_err(A3[f], B3[f]) <= stored_tol(B3[f], lim * 10), f
    for f in ("temp0", "concn0"):
        assert rel_err(A2[f], B2[f]) <= stored_tol(B2[f], lim), f
    fluid = B["p_type"] == 1
    if THERMAL[name][0]:
        assert np.abs(B3["dtemp"][fluid]).max() > 0
    if THERMAL[name][2]:
        assert np.abs(B3["dconcn"][fluid]).max() > 0


@pytest.mark.parametrize("precision,tol", [(layout.PREC_MIXED, FP32_TOL), (layout.PREC_FP64, FP64_TOL)],
                         ids=["fp32", "fp64"])
def test_enthalpy_form_step_matches_oracle(precision, tol):
    """enthalpy_eqn = 1 (the reference's compiled-out enthalpy form; the
    oracle is bit-exact against the reference built with it,
    tests/test_oracle.py): the enthalpy rate, enthalpy0, the htoT
    temperature and the enthalpy update within the step bar."""
    P, p = decks.enthalpy_mini()
    A, A2, A3, B, B2, B3 = _run_pair(P, p, precision, nsteps=3)
    lim = FP64_MOST_TOL if precision == layout.PREC_FP64 else tol
    errs = {f: rel_err(A[f], B[f]) for f in FIELDS + ["concn", "enthalpy"]}
    bad = {f: e for f, e in errs.items() if e > lim}
    assert not bad, bad
    assert rel_err(A3["denthalpy"], B3["denthalpy"]) <= stored_tol(B3["denthalpy"], lim * 10)
    assert rel_err(A2["enthalpy0"], B2["enthalpy0"]) <= stored_tol(B2["enthalpy0"], lim)
    assert np.abs(B3["denthalpy"][B["p_type"] == 1]).max() > 0


BOUNDARY = {"extrapolation": (layout.OUTLET_EXTRAPOLATION, 0), "inout": (layout.OUTLET_INOUT, 0),
            "recycling_probe": (layout.OUTLET_DONOTHING, 1), "inout_recycling_probe": (layout.OUTLET_INOUT, 1)}


@pytest.mark.parametrize("precision,tol", [(layout.PREC_MIXED, FP32_TOL), (layout.PREC_FP64, FP64_TOL)],
                         ids=["fp32", "fp64"])
@pytest.mark.parametrize("name", list(BOUNDARY))
def test_dormant_boundary_passes_match_oracle(name, precision, tol):
    """The reference's commented-out open-boundary passes (outlet
    extrapolation, inflow/outflow, inlet recycling), switched in at their call
    sites; the oracle is bit-exact against the reference for them
    (tests/test_oracle.py).  The recycling probe sits on a MOST record of the
    deck, so its friction velocity drives the inlet."""
    P, p = decks.caseh_mini(nx=12, ny=12, nz=5)
    p.outlet_bc, p.inlet_recycling = BOUNDARY[name]
    if p.inlet_recycling:
        k = int(np.nonzero(P["MOST_buffer"] == 1)[0][0])
        p.recycle_probe_x, p.recycle_probe_y = float(P["x"][k]), float(P["y"][k])
    A, A2, A3, B, B2, B3 = _run_pair(P, p, precision, nsteps=3)
    lim = FP64_MOST_TOL if precision == layout.PREC_FP64 else tol
    errs = {f: rel_err(A[f], B[f]) for f in FIELDS}
    bad = {f: e for f, e in errs.items() if not e <= lim}
    assert not bad, bad
    if p.inlet_recycling:
        inlet = B["buffer_type"] == 1
        assert np.abs(B["ux"][inlet]).max() > 0


@pytest.mark.parametrize("form", [0, 1], ids=["active_form", "difference_form"])
@pytest.mark.parametrize("precision,tol", [(layout.PREC_MIXED, FP32_TOL), (layout.PREC_FP64, FP64_TOL)],
                         ids=["fp32", "fp64"])
def test_stored_pair_factors_match_full_evaluation(precision, tol, form):
    """The prep pass and the pressure force with their time-invariant pair
    factors stored at the neighbour build (default) against the same passes
    evaluating every pair term each step (recompute_pairs = 1, the
    reference's way), and switching between the two inside a run; with the
    pressure force's active pair term and its difference form."""
    P, p = decks.caseh_mini(turbulence="DDF", seed=5)
    p.pressure_force_form = form
    out = []
    for rp in (0, 1):
        q = p.copy()
        q.ppe_mode = layout.PPE_REF_SWEEP
        q.recompute_pairs = rp
        sim = abi.Simulation(q, precision=precision)
        sim.upload(P)
        for _ in range(2):
            sim.step(1)
        q2 = q.copy()
        q2.recompute_pairs = 1 - rp
        sim.set_params(q2)
        sim.step(1)
        A, A2, A3 = sim.download()
        sim.close()
        out.append((A, A2, A3))
    (A, A2, A3), (B, B2, B3) = out
    for f in FIELDS:
        assert rel_err(A[f], B[f]) <= tol, f
    for f in ("fpx", "fpy", "fpz"):
        assert rel_err(A3[f], B3[f]) <= stored_tol(B3[f], tol * 10), f
    assert rel_err(A2["SR"], B2["SR"]) <= stored_tol(B2["SR"], tol * 10)
