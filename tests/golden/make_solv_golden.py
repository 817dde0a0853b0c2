"""Writes tests/golden/solv_ref.npz, the reference's host set-up run through
its host build in oracle/_ref:

* solver input files in the reference's keyword format and the k_vii /
  k_vif tables and plot labels its read_solv_input makes of them, each
  starting from the same seeded tables so that untouched and cleared slots
  are checked too;
* seeded deck records (every p_type class, heights below, inside and above
  the profile tables, positions on both sides of every buffer plane) and the
  records its c_initial_inner_outer_particle_single makes of them, for
  open and closed boundaries in 3-D and for 2-D.

Run from the repository root:

    python tests/golden/make_solv_golden.py
"""
import ctypes
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "urban-sph_a100_b200"), os.path.join(ROOT, "oracle")]

import refhost  # noqa: E402
from sph_b200 import decks  # noqa: E402

# An urban-canopy ISPH input: every keyword once, values in the forms the
# parser reads (the keyword, its fixed number of tokens, the value last).
FULL = """\
solver_type : ISPH
dimension(1/2/3): 3
property_table(YES/NO): NO
atmospheric-stability : Neutral
terrain-type : City
kernel type : Wendland6
time integration : Euler
structure solve: NO
open boundary type: OPEN
pressure-force : YES
viscous-force : Cleary
turbulence-model : DDF
gravitational-force : NO
Conduction(YES/NO): NO
Boussinesq-natural-convection : NO
Concentration-diffusion(YES/NO): NO
kernel-gradient-correction : KGC
switch_ptype : NO
noslip_boundary : YES
APR_solve : Cell
Block_configuration NBI: 4 NBJ: 2 NBK: 3
Variable h: Abrupt
Buffersize: 0.35
reference-pressure : 101325.0
kappa: 2.0
minimum-iteration: 3
maximum-iteration: 40
pressure-convergence : 1e-6
density-convergence : 0.001
pressure-relaxation : 0.5
time-step : 2.5e-5
start-time : 0.0
end-time : 12.5
neighbor search cell : 3X3
timestep update : NO
structure-timestep : 1e-6
filtering : 20
temperature-filtering : 50
plot-output : 400
APR_frequency: 100
h-reset : 1000
BAPR_frequency: 7
plot-variables: 6 velocity pressure p_type rho_ref i_type turbulence
velocity-limit : 15.0
"""

# A second set of choices for every enumerated switch, keywords reordered.
ALT = """\
velocity-limit : 3.5
kernel type : Quartic
time integration : Predictor_Corrector
solver_type : WCSPH
atmospheric-stability : Stable
terrain-type : Forest
open boundary type: PERIODIC
viscous-force : Violeau
turbulence-model : k-e
kernel-gradient-correction : DFPM
APR_solve : Block
Variable h: Smooth
neighbor search cell : 5X5
timestep update : YES
pressure-force : NO
gravitational-force : YES
structure solve: YES
property_table(YES/NO): YES
Conduction(YES/NO): YES
Boussinesq-natural-convection : YES
Concentration-diffusion(YES/NO): YES
switch_ptype : YES
noslip_boundary : NO
dimension(1/2/3): 2
plot-variables: 2 temp mass
"""

# Names the parser does not know leave the slot as it was; values that
# are themselves keywords start that keyword's read (the value "open" of
# "kernel" below); a keyword that is the last token of the file reads past
# the end and takes the value of its own name.
QUIRKS = """\
kernel type : Cubic
turbulence-model : Smagorinsky
kernel type : open boundary : PERIODIC
viscous-force : Monaghan
time-step : 1e-3 # comment tokens are plain tokens
maximum-iteration:
"""

CASES = {"full": FULL, "alt": ALT, "quirks": QUIRKS, "empty": "\n"}


def init_records(rng):
    """Deck records as read_input leaves them, spread over every class."""
    P, _ = decks.caseh_mini(nx=10, ny=6, nz=5)
    P = P[:600].copy()
    n = len(P)
    P["p_type"] = rng.choice(np.array([-1, 0, 1, 2, 3, 1000, -2, 9], np.int32), n)
    P["x"] = rng.uniform(-0.05, 13.4, n).astype(np.float32)
    P["x"][:40] = np.float32(13.304) + rng.integers(-2, 3, 40).astype(np.float32) * np.float32(1e-6)
    P["x"][40:80] = np.float32(0.028) + rng.integers(-2, 3, 40).astype(np.float32) * np.float32(1e-6)
    P["y"] = rng.uniform(-0.5, 0.5, n).astype(np.float32)
    P["y"][80:120] = np.float32(0.412) * rng.choice(np.array([-1, 1], np.float32), 40)
    P["z"] = rng.uniform(-0.1, 1.0, n).astype(np.float32)
    P["z"][120:140] = np.float32(0.005)
    P["z"][140:160] = np.float32(0.8919544)
    P["z"][160:170] = np.float32(0.74209)
    P["m"] = rng.uniform(0.5, 2.0, n).astype(np.float32)
    P["ux"] = rng.standard_normal(n).astype(np.float32)
    P["uy"] = rng.standard_normal(n).astype(np.float32)
    P["rho"] = rng.uniform(1.0, 1.5, n).astype(np.float32)
    P["i_type"] = 1
    return P


def main():
    L = refhost.lib()
    L.ref_read_solv.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    rng = np.random.default_rng(20)
    vii0 = rng.integers(-9, 9, 64).astype(np.int32)
    vif0 = rng.standard_normal(32).astype(np.float32)
    out = {"vii0": vii0, "vif0": vif0, "names": np.array(sorted(CASES))}
    with tempfile.TemporaryDirectory() as tmp:
        for name in sorted(CASES):
            path = os.path.join(tmp, name + ".txt")
            with open(path, "w") as f:
                f.write(CASES[name])
            vii, vif = vii0.copy(), vif0.copy()
            labels = ctypes.create_string_buffer(400)
            n = L.ref_read_solv(path.encode(), vii.ctypes.data, vif.ctypes.data, labels)
            out["text_" + name] = np.frombuffer(CASES[name].encode(), np.uint8)
            out["vii_" + name] = vii
            out["vif_" + name] = vif
            out["nlab_" + name] = np.int32(n)
            out["labels_" + name] = np.frombuffer(labels.raw, np.uint8)
    L.ref_initial_records.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    P = init_records(rng)
    out["init_in"] = P.view(np.uint8)
    for tag, open_b, dim in (("open3", 1, 3), ("closed3", 0, 3), ("open2", 1, 2)):
        Q = P.copy()
        L.ref_initial_records(Q.ctypes.data, len(Q), open_b, dim)
        out["init_" + tag] = Q.view(np.uint8)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "solv_ref.npz"), **out)
    print("wrote tests/golden/solv_ref.npz")


if __name__ == "__main__":
    main()
