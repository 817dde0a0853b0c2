"""Particle decks and VTK files in the reference's formats (host code, no GPU).

Pinned to the reference through tests/golden/io_ref.npz (made by
tests/golden/make_io_golden.py from the reference's own read_input and
save_vtk_bin_single_flag, compiled for the host): the records read from the
deck are bit-identical and the VTK file is byte-identical.  The VTK is also
parsed back independently of the reference.
"""
import os

import numpy as np
import pytest

from sph_b200 import abi, layout

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "io_ref.npz"))


def test_read_deck_matches_reference_reader(tmp_path):
    path = tmp_path / "deck.txt"
    path.write_bytes(G["deck"].tobytes())
    P = abi.read_deck(path)
    R = G["records"].view(layout.PART1)
    assert len(P) == len(R)
    assert P.tobytes() == R.tobytes()


def test_write_vtk_matches_reference_writer(tmp_path):
    Q = G["vtk_records"].view(layout.PART1)
    Q2 = G["vtk_p2"].view(layout.PART2)
    labels = G["labels"].tobytes().decode().split()
    out = tmp_path / "fluid.vtk"
    abi.write_vtk(out, Q, labels, P2=Q2)
    assert out.read_bytes() == G["vtk"].tobytes()


def _parse_vtk(data):
    """Minimal reader of the legacy binary POLYDATA the writer emits."""
    pos = 0

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode()
        pos = e + 1
        return s

    for _ in range(4):
        line()
    _, npts, _ = line().split("\t")
    npts = int(npts)
    pts = np.frombuffer(data, ">f4", npts * 3, pos).reshape(npts, 3)
    pos += npts * 12
    line()
    nf = int(line().split("\t")[1])
    arrays = {}
    while pos < len(data):
        name, nc, n, typ = line().split("\t")
        nc, n = int(nc), int(n)
        dt = ">i4" if typ == "int" else ">f4"
        arrays[name] = np.frombuffer(data, dt, n * nc, pos).reshape(n, nc)
        pos += n * nc * 4
    return pts, nf, arrays


def test_vtk_round_trip(tmp_path):
    Q = G["vtk_records"].view(layout.PART1)
    out = tmp_path / "f.vtk"
    abi.write_vtk(out, Q, ["velocity", "pressure", "p_type", "monitor"])
    pts, nf, arrays = _parse_vtk(out.read_bytes())
    sel = (Q["i_type"] == 1) | (Q["i_type"] == 2)
    assert nf == 4 and len(pts) == sel.sum()
    assert np.array_equal(pts[:, 0], Q["x"][sel]) and np.array_equal(pts[:, 2], Q["z"][sel])
    assert np.array_equal(arrays["velocity"][:, 1], Q["uy"][sel])
    assert np.array_equal(arrays["pressure"][:, 0], Q["pres"][sel])
    assert np.array_equal(arrays["p_type"][:, 0], Q["p_type"][sel])
    assert np.array_equal(arrays["monitor"][:, 0], Q["float1"][sel])


def test_label_that_needs_part2_is_rejected_without_it(tmp_path):
    Q = G["vtk_records"].view(layout.PART1)
    import pytest
    with pytest.raises(abi.SphError):
        abi.write_vtk(tmp_path / "x.vtk", Q, ["rho_ref"])


S = np.load(os.path.join(HERE, "golden", "solv_ref.npz"))


def test_read_solv_matches_reference_parser(tmp_path):
    """Every k_vii / k_vif slot and plot label equals what the reference's
    read_solv_input made of the same file from the same starting tables."""
    for name in S["names"]:
        name = str(name)
        path = tmp_path / (name + ".txt")
        path.write_bytes(S["text_" + name].tobytes())
        p = abi.params_init()
        for k in range(64):
            p.vii[k] = int(S["vii0"][k])
        for k in range(32):
            p.vif[k] = float(S["vif0"][k])
        q, labels = abi.read_solv(path, p)
        vii = np.array(q.vii[:64], np.int32)
        vif = np.array(q.vif[:32], np.float32)
        assert np.array_equal(vii, S["vii_" + name]), (name, np.nonzero(vii != S["vii_" + name]))
        assert vif.tobytes() == S["vif_" + name].tobytes(), name
        n = int(S["nlab_" + name])
        raw = S["labels_" + name].tobytes()
        assert labels == [raw[20 * k:20 * k + 20].split(b"\0")[0].decode() for k in range(n)], name


def test_read_solv_missing_file_is_an_error(tmp_path):
    with pytest.raises(abi.SphError):
        abi.read_solv(tmp_path / "absent.txt")


def test_initial_records_match_reference_host_pass():
    """Records after the host pass equal, byte for byte, what the reference's
    c_initial_inner_outer_particle_single made of the same deck records."""
    from sph_b200 import params as sp
    P = S["init_in"].view(layout.PART1)
    for tag, open_b, dim in (("open3", 1, 3), ("closed3", 0, 3), ("open2", 1, 2)):
        p = sp.default_params(open_boundary=open_b)
        p.seti("dim", dim)
        Q = abi.initial_records(p, P)
        R = S["init_" + tag].view(layout.PART1)
        for f in layout.PART1.names:
            assert Q[f].tobytes() == R[f].tobytes(), (tag, f)


def test_initial_records_rejects_short_tables():
    from sph_b200 import params as sp
    p = sp.default_params()
    P = S["init_in"].view(layout.PART1)[:4]
    with pytest.raises(abi.SphError):
        abi.initial_records(p, P, k_table=([0.0], [1.0]))


T = np.load(os.path.join(HERE, "golden", "table_ref.npz"))


def test_read_table_matches_reference_reader(tmp_path):
    """Columns, table indices and sizes equal what the reference's read_table
    stored (in Real = float) for the same file; tests/golden/table_ref.npz is
    made by tests/golden/make_table_golden.py."""
    for name in T["names"]:
        name = str(name)
        path = tmp_path / (name + ".txt")
        path.write_bytes(T["text_" + name].tobytes())
        t = abi.read_table(path)
        assert np.array_equal(np.array(t.index[:]), T["index_" + name]), name
        assert np.array_equal(np.array(t.size[:]), T["size_" + name]), name
        for c in ("T", "h", "k", "cp", "mu"):
            col = np.ctypeslib.as_array(getattr(t, c)).astype(np.float32)
            assert col.tobytes() == T[c + "_" + name].tobytes(), (name, c)
        used = np.array(t.size[:]) > 0
        assert t.n_tables == int(used.sum()) and t.n_data == int(T["size_" + name].sum()), name


def test_read_table_columns_by_slot(tmp_path):
    path = tmp_path / "t.txt"
    path.write_bytes(T["text_two_materials"].tobytes())
    t = abi.read_table(path)
    assert t.n_tables == 2
    from sph_b200 import decks
    for k, ref in enumerate((decks.TABLE_WALL, decks.TABLE_FLUID)):
        for c in ("T", "h", "k", "cp", "mu"):
            assert np.array_equal(t.column(c, k), ref[c]), (k, c)
    u = layout.PropTables.from_columns([{c: t.column(c, k) for c in ("T", "h", "k", "cp", "mu")} for k in range(2)])
    assert bytes(u) == bytes(t)


BAD_TABLES = {
    "out_of_order": "#p_type 1\n//T\n1,2\n//h\n1,2\n#end\n",
    "skipped_slot": "#p_type 0\n//T\n1,2\n//h\n1,2\n#end\n#p_type 2\n//T\n1,2\n//h\n1,2\n#end\n",
    "no_number": "#p_type\n//T\n1,2\n#end\n",
    "unclosed": "#p_type 0\n//T\n1,2\n//h\n1,2\n",
    "no_columns": "#p_type 0\n# nothing\n#end\n",
    "ragged": "#p_type 0\n//T\n1,2,3\n//h\n1,2\n#end\n",
    "too_many_entries": "#p_type 0\n//T\n" + ",".join(["1"] * 51) + "\n#end\n",
    "eleven_tables": "".join("#p_type {}\n//T\n1,2\n#end\n".format(k) for k in range(11)),
    "column_at_end": "#p_type 0\n//T\n",
    "no_value_token": "#p_type 0\n//T\n,,,",
}


@pytest.mark.parametrize("name", list(BAD_TABLES))
def test_read_table_rejects_what_the_reference_leaves_undefined(tmp_path, name):
    path = tmp_path / "bad.txt"
    path.write_text(BAD_TABLES[name])
    with pytest.raises(abi.SphError):
        abi.read_table(path)


def test_read_table_missing_file_is_an_error(tmp_path):
    with pytest.raises(abi.SphError):
        abi.read_table(tmp_path / "absent.txt")


def test_read_table_without_tables_is_empty(tmp_path):
    path = tmp_path / "none.txt"
    path.write_text("// no tables here\n#end\n")
    t = abi.read_table(path)
    assert t.n_tables == 0 and t.n_data == 0 and not any(t.size)


def _random_table_file(rng):
    """A well-formed table file (tables 0..n-1 in order, closed, at most 50
    entries, equal-length columns) in a random spelling of the format."""
    nl = "\r\n" if rng.random() < 0.2 else "\n"
    ntab = int(rng.integers(1, 11))
    budget = 50
    out = []
    if rng.random() < 0.5:
        out.append("// generated property tables" + nl)
    for t in range(ntab):
        left = ntab - t - 1
        size = int(rng.integers(1, max(2, min(12, budget - left) + 1)))
        size = max(1, min(size, budget - left))
        budget -= size
        out.append("#p_type%s%d%s%s" % (" " * int(rng.integers(1, 3)), t,
                                         " material" if rng.random() < 0.5 else "", nl))
        cols = [c for c in ("//T", "//h", "//k", "//cp", "//mu") if rng.random() < 0.7] or ["//T"]
        trailing = rng.random() < 0.15 and size >= 2
        for c in cols:
            if rng.random() < 0.3:
                out.append("# note" + nl)
            out.append(c + (" values" if rng.random() < 0.3 else "") + nl)
            n = size - 1 if trailing else size
            vals = []
            for _ in range(n):
                form = rng.integers(0, 4)
                v = rng.normal() * 10.0 ** int(rng.integers(-3, 7))
                vals.append({0: "%d" % int(v), 1: "%.6f" % v, 2: "%.9e" % v, 3: repr(float(np.float32(v)))}[int(form)])
            sep = ", " if rng.random() < 0.3 else ","
            out.append(sep.join(vals) + ("," if trailing else "") + nl)
        out.append("#end" + nl)
    return "".join(out)


@pytest.mark.skipif(not __import__("refhost").available(), reason="reference host build absent")
def test_read_table_matches_reference_reader_on_generated_files(tmp_path):
    """60 seeded files through the reference's own read_table and this
    reader: the same columns (as stored in Real = float), indices and sizes."""
    import refhost
    rng = np.random.default_rng(2024)
    for k in range(60):
        path = tmp_path / ("gen%d.txt" % k)
        path.write_text(_random_table_file(rng), newline="")
        ref = refhost.read_table(path)
        t = abi.read_table(path)
        assert np.array_equal(np.array(t.index[:]), ref["index"]), k
        assert np.array_equal(np.array(t.size[:]), ref["size"]), k
        for c in ("T", "h", "k", "cp", "mu"):
            mine = np.ctypeslib.as_array(getattr(t, c)).astype(np.float32)
            assert mine.tobytes() == ref[c].astype(np.float32).tobytes(), (k, c)
