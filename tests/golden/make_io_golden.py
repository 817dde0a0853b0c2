"""Writes tests/golden/io_ref.npz: a particle deck in the reference's input
format, the records the reference's own read_input makes of it, and the VTK
bytes its save_vtk_bin_single_flag writes for those records (run through the
host build of the reference in oracle/_ref).  Run from the repository root:

    python tests/golden/make_io_golden.py
"""
import ctypes
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "urban-sph_a100_b200"), os.path.join(ROOT, "oracle")]

from sph_b200 import decks, layout  # noqa: E402
import refhost  # noqa: E402

CODES = (1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 26, 27, 14, 17)
LABELS = "velocity pressure p_type rho_ref smoothing monitor buffer_type i_type temp mass"
VTK_DIR = "CaseH_n10_DDF(WL6,dt=2.5e-5,KGC,IBM_WM)"   # the reference writer's hard-wired directory


def deck_text(P):
    field = {1: "x", 2: "y", 3: "z", 4: "ux", 5: "uy", 6: "uz", 7: "m", 8: "p_type", 9: "h", 10: "temp",
             11: "pres", 12: "rho", 26: "h_ref", 27: "m_ref"}
    lines = ["\t".join(str(c) for c in CODES)]
    for r in P:
        vals = []
        for c in CODES:
            if c == 8:
                vals.append(str(int(r["p_type"])))
            elif c in field:
                vals.append("%.9g" % float(r[field[c]]))
            else:
                vals.append("0")
        lines.append("\t".join(vals))
    return "\n".join(lines) + "\n"


def main():
    P, _ = decks.caseh_mini(nx=6, ny=3, nz=3)
    P = P[:400]
    text = deck_text(P)
    L = refhost.lib()
    L.ref_read_input.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p]
    L.ref_save_vtk.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "deck.txt")
        with open(path, "w") as f:
            f.write(text)
        R = np.zeros(len(P) + 8, layout.PART1)
        n = L.ref_read_input(R.ctypes.data_as(ctypes.c_void_p), len(R), path.encode())
        R = R[:n]
        # records as the step leaves them: a few buffer / dummy classes for the i_type filter
        Q = R.copy()
        Q["i_type"][::7] = 2
        Q["i_type"][::11] = 3
        Q["buffer_type"][::5] = 1
        Q["float1"] = np.arange(len(Q), dtype=np.float32)
        Q2 = np.zeros(len(Q), layout.PART2)
        Q2["rho_ref"] = np.linspace(1.0, 2.0, len(Q), dtype=np.float32)
        Q3 = np.zeros(len(Q), layout.PART3)
        cwd = os.getcwd()
        os.makedirs(os.path.join(tmp, VTK_DIR))
        os.chdir(tmp)
        try:
            L.ref_save_vtk(Q.ctypes.data_as(ctypes.c_void_p), Q2.ctypes.data_as(ctypes.c_void_p),
                           Q3.ctypes.data_as(ctypes.c_void_p), len(Q), 7, LABELS.encode())
        finally:
            os.chdir(cwd)
        with open(os.path.join(tmp, VTK_DIR, "fluid_7stp.vtk"), "rb") as f:
            vtk = f.read()
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "io_ref.npz"),
                        deck=np.frombuffer(text.encode(), np.uint8), records=R.view(np.uint8),
                        vtk_records=Q.view(np.uint8), vtk_p2=Q2.view(np.uint8), vtk=np.frombuffer(vtk, np.uint8),
                        labels=np.frombuffer(LABELS.encode(), np.uint8))
    print("wrote io_ref.npz:", n, "records,", len(vtk), "VTK bytes")


if __name__ == "__main__":
    main()
