"""Particle decks and VTK files in the reference's formats (host code, no GPU).

Pinned to the reference through tests/golden/io_ref.npz (made by
tests/golden/make_io_golden.py from the reference's own read_input and
save_vtk_bin_single_flag, compiled for the host): the records read from the
deck are bit-identical and the VTK file is byte-identical.  The VTK is also
parsed back independently of the reference.
"""
import os

import numpy as np

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
