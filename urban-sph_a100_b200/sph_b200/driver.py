"""Case runner in the shape of the reference's program.

The reference's main (SOPHIA_gpu.cu:120-141) reads ./input/solv.txt with
read_solv_input, then ISPH (ISPH.cuh:53-125) reads the particle deck, sets
the domain and the cell grid, and reserves ``buffersize * num_part`` extra
records when APR is on; c_initial_inner_outer_particle_single
(functions_NNPS.cuh:196-373) prepares the deck records on the host; ISPH_Calc (ISPH_Calc.cuh:239-528) starts the step
counter at floor(time / dt + 0.5) and steps until ``time >= time_end``,
writing the binary VTK after every step whose counter (taken before the
step's increment) is a multiple of ``freq_output`` and printing the
max |u| / max |ftotal| line every ``freq_output`` steps.

``run`` does the same through the C ABI: solver input and deck in the
reference's formats, one device context, VTK files named
``fluid_<count>stp.vtk`` in ``out_dir`` with the solver input's
plot-variables.  Settings the solver input does not carry (the PPE solver
form, the wall-model and MOST constants, the inflow profile) come from
``base`` (default: ``params.default_params()``).

The reference's main also reads the property tables of ./input/data.txt
(read_table, SOPHIA_gpu.cu:132), beside its solv.txt.  Here they are read
when the solver input sets property_table YES (the only case in which the
step reads them): from ``table_path``, else data.txt beside the solver
input.  With the enthalpy form (``--enthalpy``, the reference's
compile-time enthalpy_eqn) the records' enthalpy is set from their
temperature after the upload (KERNEL_clc_TemptoEnthalpy, the start-up
pass ISPH_Calc.cuh:480-482 keeps commented out), since decks carry
temperatures only.

    python -m sph_b200.driver solv.txt deck.txt out_dir [--steps N] [--table data.txt] [--enthalpy]
        [--ppe sweep|bicgstab|mixed|gmres|idrs] [--tol X] [--coarse B] [--coarse-max M] [--coef-half]
        [--device-control] [--pair-h] [--pforce-difference]

The solver options (``solver_params``) set what the solver input cannot
carry, as the native runner's do (urban-sph_a100_b200/csrc/sophia_b200.cpp).
"""
import argparse
import math
import os
import time as _wall

import numpy as np

from . import abi, params as _params
from .layout import PART1


# deck columns: the variable codes read_input (function_init.cuh:522-548)
# understands for the fields a deck carries
DECK_CODES = (1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 26, 27)
_DECK_FIELDS = {1: "x", 2: "y", 3: "z", 4: "ux", 5: "uy", 6: "uz", 7: "m", 8: "p_type", 9: "h", 10: "temp",
                11: "pres", 12: "rho", 26: "h_ref", 27: "m_ref"}


def write_deck(path, P1):
    """Writes records in the particle-deck format of read_input: a line of
    tab-separated variable codes, then one line per record (p_type as an
    integer, every other value with nine significant digits, enough to
    round-trip an FP32 value)."""
    cols = [_DECK_FIELDS[c] for c in DECK_CODES]
    with open(path, "w") as f:
        f.write("\t".join(str(c) for c in DECK_CODES) + "\n")
        data = [np.asarray(P1[c]) for c in cols]
        for k in range(len(P1)):
            f.write("\t".join(str(int(v[k])) if c == "p_type" else "%.9g" % float(v[k])
                              for c, v in zip(cols, data)) + "\n")


_KERNEL_NAMES = {0: "Gaussian", 1: "Quintic", 2: "Quartic", 3: "Wendland2", 4: "Wendland4", 5: "Wendland6"}
_TURB_NAMES = {0: "Laminar", 1: "k-lm", 2: "k-e", 3: "HB", 4: "SSM", 5: "DDF"}


def write_solv(path, p, labels=("velocity", "pressure", "p_type")):
    """Writes the keywords of read_solv_input (function_init.cuh:166-463)
    that carry p's solver settings: kernel, time integration, open
    boundary, force switches, turbulence model, no-slip walls, APR switch
    and buffer size, kappa, time step, start and end time, filter and
    output frequencies, plot variables and the velocity limit."""
    yes = lambda v: "YES" if v else "NO"
    lines = [
        "solver_type : ISPH",
        "dimension(1/2/3): %d" % p.geti("dim"),
        "kernel type : %s" % _KERNEL_NAMES[p.geti("kernel_type")],
        "time integration : %s" % ("Predictor_Corrector" if p.geti("time_type") == 1 else "Euler"),
        "open boundary type: %s" % {1: "OPEN", 2: "PERIODIC"}.get(p.geti("open_boundary"), "NO"),
        "pressure-force : %s" % yes(p.geti("fp_solve")),
        "viscous-force : %s" % {1: "Cleary", 2: "Monaghan"}.get(p.geti("fv_solve"), "NO"),
        "turbulence-model : %s" % _TURB_NAMES[p.geti("turbulence_model")],
        "gravitational-force : %s" % yes(p.geti("fg_solve")),
        "kernel-gradient-correction : %s" % yes(p.geti("kgc_solve")),
        "noslip_boundary : %s" % yes(p.geti("noslip_bc")),
        "APR_solve : %s" % ("Cell" if p.geti("apr_solv") else "NO"),
        "Buffersize: %.9g" % p.getf("buffersize"),
        "kappa: %.9g" % p.getf("kappa"),
        "time-step : %.9g" % p.getf("dt"),
        "start-time : %.9g" % p.getf("time"),
        "end-time : %.9g" % p.getf("time_end"),
        "filtering : %d" % max(p.geti("freq_filt"), 1),
        "plot-output : %d" % max(p.geti("freq_output"), 1),
        "plot-variables: %d %s" % (len(labels), " ".join(labels)),
        "velocity-limit : %.9g" % p.getf("u_limit"),
    ]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def setup(solv_path, deck_path, base=None):
    """Parameters, plot labels and records (with APR headroom) of a case."""
    p = base.copy() if base is not None else _params.default_params()
    p, labels = abi.read_solv(solv_path, p)
    P1 = abi.read_deck(deck_path)
    abi.domain_setup(p, P1)
    P1 = abi.initial_records(p, P1)   # ISPH_Calc.cuh:386
    n = len(P1)
    extra = int(p.getf("buffersize") * n) if p.geti("apr_solv") else 0   # ISPH.cuh:116
    if extra > 0:
        D = np.zeros(extra, dtype=PART1)
        D["i_type"] = 3
        for f in ("x", "y", "z", "h", "h_ref", "m", "m_ref", "rho", "vol"):
            D[f] = P1[f][0]
        P1 = np.concatenate([P1, D])
    p.seti("num_part", n)
    p.seti("num_part2", len(P1))
    dt = np.float32(p.getf("dt"))
    p.seti("count", int(math.floor(float(np.float32(p.getf("time")) / dt) + 0.5)))   # ISPH_Calc.cuh:256
    return p, labels, P1


PPE_MODES = {"sweep": 0, "bicgstab": 1, "mixed": 2, "gmres": 4, "idrs": 5}   # SPH_PPE_*


def solver_params(ppe=None, tol=None, coarse=0, coarse_max=0, coef_half=False, device_control=False,
                  pair_h=False, pforce_difference=False, enthalpy=False):
    """Default parameters with the solver settings a solver input does not
    carry: the PPE form and tolerance, the two-level preconditioner (coarse
    blocks of B^3 cells, -B balanced by row count, at most coarse_max
    aggregates), FP16 coefficients, device-controlled solves, the
    pair-averaged h, the difference form of the pressure force, the
    enthalpy form."""
    p = _params.default_params()
    if ppe is not None:
        p.ppe_mode = PPE_MODES[ppe]
    if tol is not None and tol > 0:
        p.ppe_tol = tol
    p.ppe_coarse_block = int(coarse)
    p.ppe_coarse_max = int(coarse_max)
    if coef_half:
        p.ppe_coef_half = 1
    if device_control:
        p.ppe_refinement = 4
    if pair_h:
        p.ppe_pair_h = 1
    if pforce_difference:
        p.pressure_force_form = 1
    if enthalpy:
        p.enthalpy_eqn = 1
    return p


def read_tables(solv_path, p, table_path=None):
    """The property tables of a case (a PropTables), or None when its
    parameters do not ask for them (vii[prop_table] = 0)."""
    if p.geti("prop_table") != 1:
        return None
    path = table_path if table_path is not None else os.path.join(os.path.dirname(os.path.abspath(solv_path)),
                                                                   "data.txt")
    if not os.path.exists(path):
        raise FileNotFoundError("property_table YES needs the table file %s" % path)
    return abi.read_table(path)


def run(solv_path, deck_path, out_dir=None, base=None, precision=0, max_steps=None, log=print, table_path=None):
    """Steps a case from its solver input and deck; returns (steps, final records)."""
    p, labels, P1 = setup(solv_path, deck_path, base)
    tables = read_tables(solv_path, p, table_path)
    if out_dir is not None:
        os.makedirs(out_dir, exist_ok=True)
    freq = max(p.geti("freq_output"), 1)
    dt = np.float32(p.getf("dt"))
    t = np.float32(p.getf("time"))
    t_end = np.float32(p.getf("time_end"))
    count = p.geti("count")
    sim = abi.Simulation(p, precision=precision)
    try:
        if tables is not None:
            sim.set_prop_tables(tables)
        sim.upload(P1)
        if p.enthalpy_eqn and p.geti("con_solve") == 1:
            sim.enthalpy_from_temperature()
        wall0 = _wall.perf_counter()
        steps = 0
        while True:
            sim.step(1)
            if out_dir is not None and count % freq == 0:
                Q1, Q2, Q3 = sim.download()
                abi.write_vtk(os.path.join(out_dir, "fluid_%dstp.vtk" % count), Q1, labels, P2=Q2, P3=Q3)
            t = np.float32(t + dt)
            count += 1
            steps += 1
            if count % freq == 0 and log is not None:
                umax, _, fmax = sim.diagnostics()
                log("Simulation time: %5.2f sec" % t)
                log("Computing time: %5.2f sec" % (_wall.perf_counter() - wall0))
                log("%d\t tu_max=%5.2f\tftotal_max=%5.5f" % (count, umax, fmax))
            if t >= t_end or (max_steps is not None and steps >= max_steps):
                break
        P_final, _, _ = sim.download(want=(1,))
        return steps, P_final
    finally:
        sim.close()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("solv")
    ap.add_argument("deck")
    ap.add_argument("out_dir")
    ap.add_argument("--steps", type=int, default=None, help="stop after this many steps")
    ap.add_argument("--fp64", action="store_true", help="FP64 context instead of FP32")
    ap.add_argument("--table", default=None, help="property tables (default: data.txt beside the solver input)")
    ap.add_argument("--enthalpy", action="store_true",
                    help="energy equation in enthalpy (with Conduction YES), enthalpy set from temperature")
    ap.add_argument("--ppe", choices=sorted(PPE_MODES), default=None, help="pressure solve (default mixed)")
    ap.add_argument("--tol", type=float, default=None, help="relative residual of the solve (default 1e-6)")
    ap.add_argument("--coarse", type=int, default=0,
                    help="two-level preconditioner on B^3-cell blocks (-B: balanced by row count)")
    ap.add_argument("--coarse-max", type=int, default=0, help="most balanced aggregates")
    ap.add_argument("--coef-half", action="store_true", help="FP16 row-scaled coefficients")
    ap.add_argument("--device-control", action="store_true", help="each solve one graph under device control")
    ap.add_argument("--pair-h", action="store_true", help="pair-averaged h in the pressure rows")
    ap.add_argument("--pforce-difference", action="store_true", help="difference form of the pressure force")
    a = ap.parse_args(argv)
    base = solver_params(a.ppe, a.tol, a.coarse, a.coarse_max, a.coef_half, a.device_control, a.pair_h,
                         a.pforce_difference, a.enthalpy)
    run(a.solv, a.deck, a.out_dir, base=base, precision=1 if a.fp64 else 0, max_steps=a.steps, table_path=a.table)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
