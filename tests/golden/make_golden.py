"""Generates tests/golden/caseh_mini_ref.npz from the reference's own host
build (oracle/_ref, compiled from the reference sources by oracle/Makefile).

The fixture holds the input deck, the parameters, the reference's NNPS arrays
and the particle state after two reference steps (PPE and Neumann with
race-free snapshot semantics), so the oracle can be checked against the
reference where the reference tree is absent.  Run from the repository root:
    python tests/golden/make_golden.py
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "urban-sph_a100_b200"), os.path.join(ROOT, "oracle")]

from sph_b200 import decks  # noqa: E402
import refhost  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "caseh_mini_ref.npz")
FIELDS = ["ux", "uy", "uz", "pres", "vis_t", "flt_s", "fbx", "fby", "fbz", "fmx", "fmy", "hmz",
          "float1", "float2", "float3", "temp", "concentration"]


def main():
    P, p = decks.caseh_mini(nx=14, ny=7, nz=5)
    R = refhost.RefHost(P, p, parallel=False)
    SP1, g_idx, p_idx, g_str, g_end = R.nnps()
    R.step(2)
    out = {"deck": P.view(np.uint8), "params": np.frombuffer(bytes(p), np.uint8),
           "g_idx": g_idx, "p_idx": p_idx, "g_str": g_str, "g_end": g_end}
    for f in FIELDS:
        out["p1_" + f] = R.P1[f].copy()
    np.savez_compressed(OUT, **out)
    print(OUT, os.path.getsize(OUT), "bytes,", len(P), "particles")


if __name__ == "__main__":
    main()
