"""Writes tests/golden/table_ref.npz: property-table files in the reference's
data.txt format and the tables its read_table (function_init.cuh:724-905)
makes of them, through the reference's host build in oracle/_ref.

Each file is well formed in the sense the reference's arrays are defined
for (tables numbered 0, 1, ... in file order, every table closed by #end,
at most 50 entries in all); the forms the parser meets inside that are
covered: all five columns and subsets, comment and unknown lines inside and
outside tables, spaces around values, a trailing comma, a line of commas
only, CRLF line ends, a line longer than the 999 characters one fgets
reads, exactly 50 entries in ten tables.

Run from the repository root:

    python tests/golden/make_table_golden.py
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "urban-sph_a100_b200"), os.path.join(ROOT, "oracle")]

import refhost  # noqa: E402
from sph_b200 import decks  # noqa: E402


def _line(vals):
    return ",".join(repr(float(v)) for v in vals) + "\n"


def _table(num, cols, head="#p_type {} material\n", extra=""):
    out = head.format(num) + extra
    for key, vals in cols:
        out += key + "\n" + _line(vals)
    return out + "#end\n"


# the two-material enthalpy tables of the parity decks (decks.TABLE_WALL,
# decks.TABLE_FLUID): p_type 0 (walls, four points) and 1 (fluid, six
# points); h ascending in both
WALL, FLUID = decks.TABLE_WALL, decks.TABLE_FLUID


def two_materials():
    text = "// property tables\n\n"
    for num, t in ((0, WALL), (1, FLUID)):
        text += _table(num, [("//T", t["T"]), ("//h", t["h"]), ("//k", t["k"]), ("//cp", t["cp"]),
                             ("//mu", t["mu"])], extra="# a comment line inside\n")
    return text


def files():
    rng = np.random.default_rng(7)
    out = {"two_materials": two_materials()}
    # h and T only, values with spaces after the commas and an exponent form
    t = "#p_type 0\n//h values\n -554932, 215789 , 7.57894e5,905263\n//T\n280,1537,2300,2450\n#end\n"
    out["subset_spaced"] = t
    # a trailing comma adds an entry atof("\n") = 0 to every column line
    out["trailing_comma"] = ("#p_type 0\n//T\n1,2,3,\n//h\n10,20,30,\n#end\n"
                             "#p_type 1\n//T\n5,6\n//h\n50,60\n#end\n")
    # a value line of commas only holds one token, "\n": one entry 0
    out["commas_only"] = "#p_type 0\n//T\n,,,\n//h\n,,,\n#end\n"
    # CRLF line ends
    out["crlf"] = two_materials().replace("\n", "\r\n")
    # a line of 1500 characters outside the tables (fgets splits it) and
    # unknown keys inside
    out["long_line"] = ("x" * 1500 + "\n" + "#p_type 0\n//q ignored\n1,2\n//T\n1,2,3\n//h\n4,5,6\n"
                        "//k\n7,8,9\n#end\n")
    # ten tables of five entries: every slot and all 50 entries
    ten = ""
    for num in range(10):
        h = np.sort(rng.uniform(-1e6, 1e6, 5))
        T = np.sort(rng.uniform(250, 3000, 5))
        ten += _table(num, [("//T", T), ("//h", h), ("//k", rng.uniform(0, 5, 5)),
                            ("//cp", rng.uniform(100, 900, 5)), ("//mu", rng.uniform(0, 1e-2, 5))])
    out["ten_tables"] = ten
    return out


def main():
    data = {}
    names = []
    with tempfile.TemporaryDirectory() as d:
        for name, text in files().items():
            path = os.path.join(d, name + ".txt")
            with open(path, "wb") as f:
                f.write(text.encode())
            r = refhost.read_table(path)
            names.append(name)
            data["text_" + name] = np.frombuffer(text.encode(), np.uint8)
            for c in ("T", "h", "k", "cp", "mu"):
                data[c + "_" + name] = r[c].astype(np.float32)   # stored in Real = float
            data["index_" + name] = r["index"]
            data["size_" + name] = r["size"]
    data["names"] = np.array(names)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "table_ref.npz"), **data)
    print("wrote tests/golden/table_ref.npz:", ", ".join(names))


if __name__ == "__main__":
    main()
