"""The case runner: solver input + particle deck in the reference's formats
through set-up, stepping and VTK output (set-up on the CPU, the run on the
GPU)."""
import json
import os
import subprocess

import numpy as np
import pytest

from sph_b200 import abi, decks, driver, layout

SOLV = """\
solver_type : ISPH
dimension(1/2/3): 3
kernel type : Wendland6
time integration : Predictor_Corrector
open boundary type: OPEN
pressure-force : YES
viscous-force : Cleary
turbulence-model : SSM
gravitational-force : NO
kernel-gradient-correction : NO
noslip_boundary : YES
APR_solve : {apr}
Buffersize: 0.25
kappa: 2.0
time-step : 1e-4
start-time : {t0}
end-time : 1.0
filtering : 1
plot-output : 2
plot-variables: 3 velocity pressure p_type
velocity-limit : 50.0
"""

CODES = (1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 26, 27)
FIELDS = {1: "x", 2: "y", 3: "z", 4: "ux", 5: "uy", 6: "uz", 7: "m", 8: "p_type", 9: "h", 10: "temp",
          11: "pres", 12: "rho", 26: "h_ref", 27: "m_ref"}


def write_case(tmp_path, apr="NO", t0="0.0"):
    P, _ = decks.caseh_mini()
    lines = ["\t".join(str(c) for c in CODES)]
    for r in P:
        lines.append("\t".join(str(int(r["p_type"])) if c == 8 else "%.9g" % float(r[FIELDS[c]])
                               for c in CODES))
    deck = tmp_path / "deck.txt"
    deck.write_text("\n".join(lines) + "\n")
    solv = tmp_path / "solv.txt"
    solv.write_text(SOLV.format(apr=apr, t0=t0))
    return solv, deck, P


def test_setup_reads_solver_input_and_deck(tmp_path):
    solv, deck, P = write_case(tmp_path)
    p, labels, Q = driver.setup(solv, deck)
    assert labels == ["velocity", "pressure", "p_type"]
    assert p.geti("solver_type") == 1 and p.geti("time_type") == 1 and p.geti("open_boundary") == 1
    assert p.geti("freq_output") == 2 and p.getf("dt") == np.float32(1e-4)
    assert len(Q) == len(P) and p.geti("num_part2") == len(P) and p.geti("count") == 0
    # the host pass ran: buffer classes assigned, m_ref = m, temp 300
    assert (Q["i_type"] == 2).sum() > 0
    assert np.array_equal(Q["m_ref"], Q["m"]) and np.all(Q["temp"] == np.float32(300.0))
    assert p.geti("NI") > 0 and p.geti("num_cells") == p.geti("NI") * p.geti("NJ") * p.geti("NK") + 1


def test_setup_reserves_apr_headroom_and_restart_count(tmp_path):
    solv, deck, P = write_case(tmp_path, apr="Cell", t0="0.0025")
    p, _, Q = driver.setup(solv, deck)
    extra = int(np.float32(0.25) * len(P))
    assert len(Q) == len(P) + extra and p.geti("num_part") == len(P)
    assert np.all(Q["i_type"][len(P):] == 3)
    assert p.geti("count") == 25          # floor(time / dt + 0.5)


@pytest.mark.gpu
def test_run_writes_reference_vtk_series(tmp_path):
    solv, deck, _ = write_case(tmp_path)
    out = tmp_path / "out"
    log = []
    steps, P = driver.run(solv, deck, out, max_steps=3, log=log.append)
    assert steps == 3
    names = sorted(os.listdir(out))
    assert names == ["fluid_0stp.vtk", "fluid_2stp.vtk"]
    alive = np.isin(P["i_type"], (1, 2))
    assert np.all(np.isfinite(P["ux"][alive])) and np.all(np.isfinite(P["pres"][alive]))
    assert np.abs(P["ux"][alive]).max() < 50.0
    data = (out / "fluid_2stp.vtk").read_bytes()
    assert b"POINTS\t%d\tfloat" % alive.sum() in data
    assert any("tu_max" in line for line in log)


def test_written_deck_and_solver_input_read_back(tmp_path):
    """write_deck / write_solv produce files that the readers pinned to the
    reference's own parser give back unchanged: the deck's records and every
    k_vii / k_vif slot the solver input carries."""
    import refhost
    P, p = decks.canyon(scale=0.12)
    p.setf("time_end", 0.0123)
    p.seti("freq_output", 77)
    deck = tmp_path / "deck.txt"
    solv = tmp_path / "solv.txt"
    driver.write_deck(deck, P)
    driver.write_solv(solv, p)
    Q = abi.read_deck(deck)
    assert len(Q) == len(P)
    for c in ("x", "y", "z", "ux", "uy", "uz", "m", "p_type", "h", "temp", "pres", "rho", "h_ref", "m_ref"):
        assert np.array_equal(Q[c], P[c]), c
    q, labels = abi.read_solv(solv, decks.default_params())
    for slot in ("dim", "kernel_type", "time_type", "open_boundary", "fp_solve", "fv_solve", "fg_solve",
                 "kgc_solve", "turbulence_model", "noslip_bc", "apr_solv", "freq_filt", "freq_output"):
        assert q.geti(slot) == p.geti(slot), slot
    for slot in ("kappa", "dt", "time", "time_end", "u_limit", "buffersize"):
        assert np.float32(q.getf(slot)) == np.float32(p.getf(slot)), slot
    assert labels == ["velocity", "pressure", "p_type"]
    if refhost.available():
        import ctypes
        L = refhost.lib()
        L.ref_read_solv.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p]
        vii = np.zeros(64, np.int32)
        vif = np.zeros(32, np.float32)
        buf = ctypes.create_string_buffer(400)
        L.ref_read_solv(str(solv).encode(), vii.ctypes.data_as(ctypes.c_void_p),
                        vif.ctypes.data_as(ctypes.c_void_p), buf)
        from sph_b200 import layout
        for slot in ("dim", "kernel_type", "time_type", "open_boundary", "turbulence_model", "freq_output"):
            assert int(vii[layout.VII[slot]]) == p.geti(slot), slot
        for slot in ("dt", "time_end", "u_limit"):
            assert vif[layout.VIF[slot]] == np.float32(p.getf(slot)), slot


def test_property_tables_are_read_beside_the_solver_input(tmp_path):
    """property_table YES: the tables come from data.txt beside solv.txt (the
    reference's ./input layout) or from the path given; without the file the
    case is refused; with NO nothing is read."""
    solv, deck, _ = write_case(tmp_path)
    p, _, _ = driver.setup(solv, deck)
    assert driver.read_tables(solv, p) is None
    solv.write_text(solv.read_text() + "property_table(YES/NO): YES\n")
    p, _, _ = driver.setup(solv, deck)
    assert p.geti("prop_table") == 1
    with pytest.raises(FileNotFoundError):
        driver.read_tables(solv, p)
    G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "table_ref.npz"))
    (tmp_path / "data.txt").write_bytes(G["text_two_materials"].tobytes())
    t = driver.read_tables(solv, p)
    assert t.n_tables == 2 and np.array_equal(t.column("T", 1), decks.TABLE_FLUID["T"])
    other = tmp_path / "elsewhere.txt"
    other.write_bytes(G["text_ten_tables"].tobytes())
    assert driver.read_tables(solv, p, other).n_tables == 10


NATIVE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "urban-sph_a100_b200", "lib", "sophia_b200")
needs_native = pytest.mark.skipif(not os.path.exists(NATIVE), reason="native runner not built (build.py)")


def _native(*args):
    return subprocess.run([NATIVE] + [str(a) for a in args], capture_output=True, text=True, timeout=120)


@needs_native
@pytest.mark.parametrize("apr,t0", [("NO", "0.0"), ("Cell", "0.0025")])
def test_native_runner_sets_up_the_case_as_the_python_runner(tmp_path, apr, t0):
    """sophia_b200 --setup-only (solver input, deck, domain, host record
    pass, APR headroom, step counter; no device call) against driver.setup."""
    solv, deck, _ = write_case(tmp_path, apr=apr, t0=t0)
    r = _native(solv, deck, tmp_path / "out", "--setup-only")
    assert r.returncode == 0, r.stderr
    got = json.loads(r.stdout.strip().splitlines()[-1])
    p, labels, Q = driver.setup(solv, deck)
    assert got["num_part2"] == len(Q) == p.geti("num_part2") and got["num_part"] == p.geti("num_part")
    assert got["count"] == p.geti("count")
    for k in ("NI", "NJ", "NK", "num_cells"):
        assert got[k] == p.geti(k), k
    assert np.float32(got["dcell"]) == np.float32(p.getf("dcell"))
    assert got["labels"] == len(labels) and got["prop_table"] == 0 and got["tables"] == 0


@needs_native
def test_native_runner_reads_the_tables_beside_the_solver_input(tmp_path):
    solv, deck, _ = write_case(tmp_path)
    solv.write_text(solv.read_text() + "property_table(YES/NO): YES\n")
    r = _native(solv, deck, tmp_path / "out", "--setup-only")
    assert r.returncode == 1 and "data.txt" in r.stderr
    G = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "table_ref.npz"))
    (tmp_path / "data.txt").write_bytes(G["text_two_materials"].tobytes())
    r = _native(solv, deck, tmp_path / "out", "--setup-only")
    assert r.returncode == 0, r.stderr
    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert got["prop_table"] == 1 and got["tables"] == 2
    bad = tmp_path / "bad.txt"
    bad.write_text("#p_type 3\n//T\n1,2\n#end\n")
    r = _native(solv, deck, tmp_path / "out", "--setup-only", "--table", bad)
    assert r.returncode == 1 and "property tables" in r.stderr


@needs_native
def test_native_runner_rejects_bad_arguments(tmp_path):
    assert _native().returncode == 2
    assert _native("a", "b", "c", "--bogus").returncode == 2
    r = _native(tmp_path / "absent.txt", tmp_path / "deck.txt", tmp_path / "out", "--setup-only")
    assert r.returncode == 1 and "solver input" in r.stderr


@pytest.mark.gpu
@needs_native
def test_native_runner_writes_the_python_runners_files(tmp_path):
    """Three steps through sophia_b200 and through driver.run: the same VTK
    series, byte for byte (the same library, called the same way)."""
    solv, deck, _ = write_case(tmp_path)
    r = _native(solv, deck, tmp_path / "native", "--steps", 3)
    assert r.returncode == 0, r.stderr
    driver.run(solv, deck, tmp_path / "python", max_steps=3, log=None)
    names = sorted(os.listdir(tmp_path / "python"))
    assert names == sorted(os.listdir(tmp_path / "native")) == ["fluid_0stp.vtk", "fluid_2stp.vtk"]
    for f in names:
        assert (tmp_path / "native" / f).read_bytes() == (tmp_path / "python" / f).read_bytes(), f
    assert "tu_max" in r.stdout


@needs_native
@pytest.mark.parametrize("flags,kw", [
    ([], {}),
    (["--ppe", "sweep"], dict(ppe="sweep")),
    (["--ppe", "gmres", "--tol", "1e-8", "--coarse", "-16", "--coarse-max", "16384", "--coef-half",
      "--device-control", "--pair-h", "--pforce-difference", "--enthalpy"],
     dict(ppe="gmres", tol=1e-8, coarse=-16, coarse_max=16384, coef_half=True, device_control=True, pair_h=True,
          pforce_difference=True, enthalpy=True)),
])
def test_native_runner_solver_options_match_the_python_runner(tmp_path, flags, kw):
    solv, deck, _ = write_case(tmp_path)
    r = _native(solv, deck, tmp_path / "out", "--setup-only", *flags)
    assert r.returncode == 0, r.stderr
    got = json.loads(r.stdout.strip().splitlines()[-1])
    p = driver.solver_params(**kw)
    for f in ("ppe_mode", "ppe_coarse_block", "ppe_coarse_max", "ppe_coef_half", "ppe_refinement", "ppe_pair_h",
              "pressure_force_form", "enthalpy_eqn"):
        assert got[f] == getattr(p, f), f
    assert got["ppe_tol"] == p.ppe_tol


@needs_native
def test_native_runner_rejects_an_unknown_solver(tmp_path):
    solv, deck, _ = write_case(tmp_path)
    assert _native(solv, deck, tmp_path / "out", "--setup-only", "--ppe", "cg").returncode == 2
