#!/usr/bin/env python
"""Benchmark of the B200 ISPH step.

Default workload: the staggered 4x4 cube array (4.8 x 2.4 x 0.8 m, base
dx = 0.01 m) with two-level APR within 0.1 m of the cube faces, stepped in
the mixed-precision form with the learned PPE warm start, against the plain
FP64 form (Jacobi-BiCGSTAB) timed in the same run.  --config canyon / tgv /
ensemble / transfer select the other workloads.

One JSON line on rank 0:
  metric  particle-steps/s: active particles x steps / device time of the
          full step (interaction passes, PPE converged to ||b-Ap||/||b|| <=
          1e-6 with FP32 BiCGSTAB and FP64 reliable updates, time update);
          NNPS runs at step 0 inside the warm-up (the reference runs it only
          at step 0, ISPH_Calc.cuh:23-52, because particles never move).
  e2e     the same step through the C ABI with host buffers: every step
          uploads the particle records (part1, pinned host memory), runs the
          step and downloads the records again.
  roofline of the dominant kernel (the PPE operator), from live CUDA-event
          timing of its launches inside the timed region.
  plain_fp64 / error_vs_plain_fp64  the plain FP64 form on the same deck and
          the chosen form's velocity and pressure error against it.
  nnps_bit_exact  cell hash, permutation, cell ranges and neighbour lists of
          the timed deck against the CPU oracle.
  cpu_baseline  the reference's own step compiled for the host cores
          (oracle/_ref), timed on a bounded sample of the config's deck.
With --impl reference only the reference arm runs (rank 0).
Multi-GPU: the step is a one-GPU path; N ranks run N independent replicas
(weak scaling, no collective in the step).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "urban-sph_a100_b200"), os.path.join(ROOT, "oracle")]

METRIC = "particle-steps/s"
WORKLOAD = "urban canyon 2.4x1.2x0.6 m, dx=0.01 m: 240x120x60 fluid + floor walls + free-slip ceiling + IBM cube, neutral MOST, SSM Cs=0.12"
WORKLOAD_ARRAY = ("staggered 4x4 array of 0.1 m IBM cubes at 0.3 m pitch in a 4.8x2.4x0.8 m channel, base dx=0.01 m, "
                  "{res}, SSM Cs=0.12, log-law inflow u*=0.3 m/s z0=0.01 m with a seeded 5% perturbation; MOST runs "
                  "neutral: with the stable L=100 m surface temperature difference the reference's Obukhov-length "
                  "Newton iteration (functions_MOST.cuh:205-245) returns NaN at the low-wind wall-layer records of "
                  "this deck, in the reference's own kernel as here")
RES_APR = "two-level APR (ratio 2, children at dx/2) within 0.1 m of the cube faces"
RES_UNIFORM = "uniform resolution"
WORKLOAD_TGV = ("triply periodic Taylor-Green vortex: {n}^3 particles, dx=1/{n} m in a 1 m cube with 3 layers of "
                "periodic ghosts, h=1.3dx, Wendland C6, rho=1000, nu=1e-3, U0=1 m/s, CFL 0.1")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(name):
    """DRAM bytes per launch of the operator from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            d = json.load(f)
        return d
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            with open(self.path, "w") as out:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                              "--format=csv,noheader,nounits", "-lms", "200"],
                                             stdout=out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
                except ValueError:
                    continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def reference_sample(config):
    """The bounded deck on which the reference's own host step is timed, and
    its description.  The reference compiles no APR and runs one in-place
    PPE sweep per step (ISPH_Calc.cuh:137-154), so its sample is the
    uniform-resolution deck of the config at reduced extent."""
    from sph_b200 import decks
    if config == "array":
        P, p, _ = decks.cube_array(scale=0.2)
        what = (f"uniform-resolution cube array at scale 0.2 ({len(P)} particles; the reference compiles no APR), "
                f"the reference's step: one in-place PPE sweep, no converged solve")
    else:
        P, p = decks.canyon(scale=0.3)
        what = (f"canyon deck at scale 0.3 ({len(P)} particles), the reference's step: one in-place PPE sweep, "
                f"no converged solve")
    return P, p, what


def cpu_baseline(steps, config="canyon"):
    """The reference's own step on the host cores, bounded sample of the deck."""
    import refhost
    if not refhost.available():
        return None
    P, p, what = reference_sample(config)
    R = refhost.RefHost(P, p, parallel=True)
    R.step(1)   # step 0: NNPS + first step (untimed)
    t0 = time.perf_counter()
    R.step(steps)
    dt = time.perf_counter() - t0
    cores = int(refhost.lib().ref_num_threads())
    return {"value": len(P) * steps / dt, "unit": METRIC, "cores": cores, "kind": "reference",
            "sample": f"{what}; {steps} steps after its step-0 NNPS, host build of the reference kernels "
                      f"(oracle/_ref) with its hard-wired Case-H constants",
            "seconds": dt}


def cpu_converged_port(local, steps=1, pforce_form=1):
    """Like-for-like CPU work: the CPU restatement of the step in FP64 with
    Jacobi-BiCGSTAB to 1e-6 (the plain form) on the refined cube array at
    scale 0.1, split by the GPU's APR passes; one thread."""
    import restated
    from sph_b200 import abi, decks, layout
    P, p, boxes = decks.cube_array(scale=0.1, apr=True)
    p.ppe_pair_h = 1
    p.pressure_force_form = pforce_form
    sim = abi.Simulation(p, precision=layout.PREC_MIXED, device=local)
    sim.set_ib_boxes(boxes)
    sim.upload(P)
    for _ in range(16):
        if sim.apr()[0] == 0:
            break
    P, _, _ = sim.download()
    sim.close()
    n = int((P["i_type"] < 3).sum())
    q = p.copy()
    q.ppe_tol = 1e-6
    O = restated.Restated(P, q, 1)
    O.step(1, mode=layout.PPE_BICGSTAB, tol=1e-6, maxit=40000)    # NNPS and the first step, untimed
    t0 = time.perf_counter()
    st = O.step(steps, mode=layout.PPE_BICGSTAB, tol=1e-6, maxit=40000)
    dt = time.perf_counter() - t0
    return {"value": n * steps / dt, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"refined cube array at scale 0.1 ({n} active particles, one cube), {steps} step(s) of the "
                      f"CPU restatement in FP64 with Jacobi-BiCGSTAB to 1e-6 after one untimed step "
                      f"({st[2]} iterations in the last)",
            "seconds": dt}


REF_CUDA = os.path.join(ROOT, "baseline", "_ref", "sophia_gpu_sm100a")
REF_VTK_DIR = "CaseH_n10_DDF(WL6,dt=2.5e-5,KGC,IBM_WM)"   # functions_OUTPUT.cuh:142


def ref_cuda_inputs(run_dir, P, p, steps):
    """The files the reference's program reads (SOPHIA_gpu.cu:124-129,
    ISPH.cuh:59): ./input/solv.txt for `steps` steps from t = 0 with output
    only at step 0, an empty ./input/data.txt (no property tables) and the
    deck ./input/CaseH_n10.txt; plus the VTK directory its writer expects."""
    from sph_b200 import driver
    os.makedirs(os.path.join(run_dir, "input"), exist_ok=True)
    os.makedirs(os.path.join(run_dir, REF_VTK_DIR), exist_ok=True)
    q = p.copy()
    dt = float(q.getf("dt"))
    q.setf("time", 0.0)
    q.setf("time_end", dt * (steps - 0.5))
    q.seti("freq_output", 100000000)
    driver.write_solv(os.path.join(run_dir, "input", "solv.txt"), q, labels=("velocity", "pressure"))
    open(os.path.join(run_dir, "input", "data.txt"), "w").close()
    driver.write_deck(os.path.join(run_dir, "input", "CaseH_n10.txt"), P)


def ref_cuda_baseline(config, warmup, steps):
    """The reference's own CUDA program recompiled for sm_100a
    (baseline/build_ref_cuda.py), run on this config's deck in its file
    formats; wall clock of `steps` steps after `warmup` (the patched timer,
    a device synchronise on both sides).  Its step is the reference's: one
    PPE sweep, every launch followed by cudaDeviceSynchronize."""
    if not os.path.exists(REF_CUDA):
        return {"unavailable": "baseline/_ref/sophia_gpu_sm100a not built (python baseline/build_ref_cuda.py)"}
    from sph_b200 import decks
    if config == "array":
        P, p, _ = decks.cube_array(scale=1.0)
        what = "uniform-resolution cube array at full size (the reference compiles no APR)"
    else:
        P, p = decks.canyon(scale=1.0)
        what = "urban canyon at full size"
    with tempfile.TemporaryDirectory() as run_dir:
        t0 = time.perf_counter()
        ref_cuda_inputs(run_dir, P, p, warmup + steps)
        t_files = time.perf_counter() - t0
        env = dict(os.environ, SOPHIA_WARMUP=str(warmup))
        t0 = time.perf_counter()
        r = subprocess.run([REF_CUDA, "1"], cwd=run_dir, env=env, capture_output=True, text=True, timeout=1800)
        t_run = time.perf_counter() - t0
    line = [x for x in r.stdout.splitlines() if x.startswith("SOPHIA_TIMED")]
    if r.returncode != 0 or not line:
        return {"unavailable": f"reference program exit {r.returncode}: " + (r.stderr or r.stdout)[-300:]}
    kv = dict(x.split("=") for x in line[-1].split()[1:])
    k, sec = int(kv["steps"]), float(kv["seconds"])
    return {"value": len(P) * k / sec, "unit": METRIC, "ms_per_step": 1e3 * sec / k, "steps": k, "warmup": warmup,
            "particles": int(len(P)), "dtype": "f32",
            "sample": f"{what}; the reference's step (one PPE sweep) as shipped, Case-H constants, recompiled "
                      f"for sm_100a; wall clock with a device synchronise on both sides",
            "input_files_s": t_files, "process_s": t_run}


def nnps_check(P, p, boxes, local):
    """Cell hash, sort permutation, cell start/end and the neighbour lists of
    the timed deck (the records as the timed context held them after the
    APR passes) from a fresh context, against the CPU oracle on the same
    records: bit-exact or not."""
    import numpy as np
    import restated
    from sph_b200 import abi, layout
    t0 = time.perf_counter()
    sim = abi.Simulation(p, precision=layout.PREC_MIXED, device=local)
    if boxes is not None:
        sim.set_ib_boxes(boxes)
    sim.upload(P)
    sim.nnps()
    g = sim.export_nnps()
    off, lst = sim.neighbors()
    sim.close()
    O = restated.Restated(P, p, 0)
    O.nnps()
    og = O.export_nnps()
    arrays = all(np.array_equal(a, b) for a, b in zip(g, og))
    ooff, olst = O.neighbors()
    del O
    lists = bool(np.array_equal(off, ooff) and np.array_equal(lst, olst))
    return {"nnps_arrays": bool(arrays), "neighbour_lists": lists, "bit_exact": bool(arrays and lists),
            "records": int(len(P)), "list_entries": int(len(lst)), "seconds": time.perf_counter() - t0}


def form_error(A, B, u_limit):
    """Relative error of state A against state B over the fluid particles
    (active, p_type 1, not periodic ghosts): L2 and max norms of velocity and
    pressure.  The corrector keeps the predictor velocity where the corrected
    one reaches u_limit, a discontinuous rule: particles within 5 % of
    u_limit in exactly one of the two states are counted apart, and the
    velocity L2 norm over the other particles is reported beside the full
    one."""
    import numpy as np
    from sph_b200 import layout
    fl = (B["i_type"] < 3) & (B["p_type"] == 1) & (B["buffer_type"] != layout.BUFFER_PERIODIC_GHOST)
    ua = np.stack([A[f][fl] for f in ("ux", "uy", "uz")], 1).astype(np.float64)
    ub = np.stack([B[f][fl] for f in ("ux", "uy", "uz")], 1).astype(np.float64)
    pa, pb = A["pres"][fl].astype(np.float64), B["pres"][fl].astype(np.float64)
    tiny = 1e-300
    near = 0.95 * float(u_limit)
    flip = (np.linalg.norm(ua, axis=1) >= near) != (np.linalg.norm(ub, axis=1) >= near)
    rest = ~flip
    return {"particles": int(fl.sum()),
            "u_rel_l2": float(np.linalg.norm(ua - ub) / max(np.linalg.norm(ub), tiny)),
            "u_rel_max": float(np.abs(ua - ub).max(initial=0.0) / max(np.abs(ub).max(initial=0.0), tiny)),
            "p_rel_l2": float(np.linalg.norm(pa - pb) / max(np.linalg.norm(pb), tiny)),
            "p_rel_max": float(np.abs(pa - pb).max(initial=0.0) / max(np.abs(pb).max(initial=0.0), tiny)),
            "u_limit_decided_differently": int(flip.sum()),
            "u_rel_l2_other_particles": float(np.linalg.norm(ua[rest] - ub[rest]) / max(np.linalg.norm(ub[rest]), tiny))}


def cpu_baseline_tgv(steps):
    """The Taylor-Green box on the host: the reference has no triply periodic
    mode, so the CPU restatement of its step (the oracle, FP64, one thread,
    Jacobi-BiCGSTAB to 1e-8) is timed on a bounded sample of the deck."""
    import restated
    from sph_b200 import decks, layout
    n = 32
    P, p = decks.tgv_periodic(n=n)
    O = restated.Restated(P, p, 1)
    O.step(1, mode=layout.PPE_BICGSTAB, tol=1e-8, maxit=4000)   # untimed first step
    t0 = time.perf_counter()
    for _ in range(steps):
        O.step(1, mode=layout.PPE_BICGSTAB, tol=1e-8, maxit=4000)
    dt = time.perf_counter() - t0
    return {"value": n ** 3 * steps / dt, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"Taylor-Green box at {n}^3 particles (dx = 1/{n} m, same physics), {steps} steps of the "
                      f"CPU restatement of the step in FP64 with Jacobi-BiCGSTAB to 1e-8 after one untimed step; "
                      f"the reference itself has no triply periodic mode",
            "seconds": dt}


def run_ensemble(args, rank, world, local):
    """Batched ensemble: every rank steps its own seeded set of cases."""
    import numpy as np
    import torch
    from sph_b200 import abi, decks, layout, replicas
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    cases = []
    for P, p, meta in decks.ensemble(args.cases, seed=20261203 + rank):
        p.ppe_mode = layout.PPE_MIXED_IR
        p.ppe_tol = 1e-6
        p.ppe_coarse_block = 3
        p.ppe_refinement = 0 if args.host_control else 4   # each solve one graph under device control
        cases.append((P, p))
    b = abi.Batch(cases, precision=layout.PREC_MIXED, device=local)
    workers, pair_block, probe_ms = b.autotune_shapes(probe_steps=1)
    b.step(max(args.warmup - 1, 1))
    clocks = Clocks(local)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks.start()
    e0.record()
    stats = b.step(args.steps)
    torch.cuda.synchronize()
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    n = b.particles()
    # every rank steps its own seeded cases: all ranks' work over the slowest rank's time
    value, ms = replicas.throughput(n, args.steps, ms, device="cuda")
    out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
           "config": {"workload": f"batched ensemble: {args.cases} lid-driven cavity / Taylor-Green cases, "
                                  "20k-200k fluid particles each at dx = 0.01 m, Re in [100, 2000], seeded",
                      "particles": n, "cases": args.cases, "workers": workers, "pair_pass_threads": pair_block,
                      "autotune_probe_ms": probe_ms,
                      "ppe": "mixed_ir + coarse 3, " + ("host-controlled Krylov loop" if args.host_control else
                                                         "each solve one CUDA graph under device control"),
                      "parallelism": "replicas" if world > 1 else "single GPU"},
           "ppe": {"iterations_mean": float(np.mean([s.iterations for s in stats])),
                   "rel_residual_max": float(max(s.rel_residual for s in stats)),
                   "not_converged_steps": sum(1 for s in stats if s.status != 0)},
           "e2e": None, "clocks": ck}
    b.close()
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_transfer(args, rank, world, local):
    """Learned warm start across decks: the network is trained on the
    pressure solves of the urban canyon (dx = 0.01 m) and starts the solves
    of the cube-array geometry at dx = 0.0075 m.  Three forms from the same
    start on the array: the mixed form with the previous pressure as start
    vector, the same with the learned start, and the plain FP64 form (Jacobi
    BiCGSTAB), which judges both."""
    import numpy as np
    import torch
    from sph_b200 import abi, decks, layout
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    t_all = time.perf_counter()
    # ---- training on the canyon's solves ----
    P, p = decks.canyon(scale=1.0)
    p.ppe_mode, p.ppe_tol, p.ppe_coarse_block = layout.PPE_MIXED_IR, 1e-6, 5
    sim = abi.Simulation(p, precision=layout.PREC_MIXED, device=local)
    sim.upload(P)
    every = max(1, len(P) * args.train_solves // 1900000)
    sim.ml_collect(every)
    for _ in range(args.train_solves):
        sim.step(1)
    sim.ml_collect(0)
    nsamp = int(lib_sample_count(sim))
    t0 = time.perf_counter()
    loss = sim.ml_train(epochs=6, batch=4096, lr=1e-3, seed=20261203)
    train_s = time.perf_counter() - t0
    w = sim.ml_get_weights()
    sim.close()
    # ---- the array geometry at the finer spacing ----
    Pa, pa, boxes = decks.cube_array(scale=args.scale, dx=args.dx)
    pa.ppe_tol = 1e-6
    n = int((Pa["i_type"] < 3).sum())
    coarse = args.coarse if args.coarse is not None else 12

    def form(precision, mode, cb, weights, steps):
        q = pa.copy()
        q.ppe_mode, q.ppe_coarse_block = mode, cb
        sd = abi.Simulation(q, precision=precision, device=local)
        sd.set_ib_boxes(boxes)
        if weights is not None:
            sd.ml_set_weights(weights)
        sd.upload(Pa)
        for _ in range(2):
            sd.step(1)
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        st = []
        g0.record()
        for _ in range(steps):
            s_ = sd.step(1)
            st.append((s_.iterations, s_.rel_residual, s_.solve_ms, s_.initial_residual, s_.status))
        g1.record()
        torch.cuda.synchronize()
        ms = g0.elapsed_time(g1)
        A = sd.download(want=(1,))[0]
        sd.close()
        return A, {"value": n * steps / (ms / 1e3), "ms_per_step": ms / steps,
                   "ppe_iterations": float(np.mean([x[0] for x in st])),
                   "rel_residual_max": float(max(x[1] for x in st)),
                   "ppe_ms": float(np.mean([x[2] for x in st])),
                   "initial_residual_mean": float(np.mean([x[3] for x in st])),
                   "not_converged_steps": sum(1 for x in st if x[4] != 0)}

    k = args.steps
    Ap, prev = form(layout.PREC_MIXED, layout.PPE_MIXED_IR, coarse, None, k)
    Al, lrn = form(layout.PREC_MIXED, layout.PPE_LEARNED, coarse, w, k)
    A64, plain = form(layout.PREC_FP64, layout.PPE_BICGSTAB, 0, None, k)
    fl = (A64["i_type"] < 3) & (A64["p_type"] == 1)

    def err(A):
        ua = np.stack([A[f][fl] for f in ("ux", "uy", "uz")]).astype(np.float64)
        ub = np.stack([A64[f][fl] for f in ("ux", "uy", "uz")]).astype(np.float64)
        pa_, pb = A["pres"][fl].astype(np.float64), A64["pres"][fl].astype(np.float64)
        return {"u_rel_l2": float(np.linalg.norm(ua - ub) / np.linalg.norm(ub)),
                "p_rel_l2": float(np.linalg.norm(pa_ - pb) / np.linalg.norm(pb))}

    prev["error_vs_plain_fp64"] = err(Ap)
    lrn["error_vs_plain_fp64"] = err(Al)
    out = {"metric": METRIC, "value": lrn["value"], "unit": METRIC, "n_gpus": 1, "steps": k,
           "warmup": 2, "ms_per_step": lrn["ms_per_step"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
           "config": {"workload": f"learned warm start trained on the urban canyon (dx 0.01 m, {args.train_solves} "
                                  f"solves) applied to the 4x4 cube array at dx {args.dx} m",
                      "particles": n, "scale": args.scale, "coarse": coarse},
           "training": {"solves": args.train_solves, "samples": nsamp, "every_kth_fluid_row": every,
                        "loss": loss, "train_s": train_s},
           "mixed_learned": lrn, "mixed_previous_pressure": prev, "plain_fp64": plain,
           "iterations_saved_per_step": prev["ppe_iterations"] - lrn["ppe_iterations"],
           "learned_vs_plain_fp64": lrn["value"] / plain["value"],
           "wall_s": time.perf_counter() - t_all}
    print(json.dumps(out))
    return 0


def lib_sample_count(sim):
    import ctypes
    from sph_b200 import abi
    cnt = ctypes.c_int64(0)
    abi.lib().sph_ml_samples(sim.h, 0, 0, None, None, ctypes.byref(cnt))
    return cnt.value


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import refhost
    if not refhost.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsophia_ref.so not built"}))
        return 0
    P, p, what = reference_sample(args.config)
    R = refhost.RefHost(P, p, parallel=True)
    for _ in range(max(args.warmup, 1)):
        R.step(1)
    t0 = time.perf_counter()
    R.step(args.steps)
    dt = time.perf_counter() - t0
    value = len(P) * args.steps / dt
    cores = int(refhost.lib().ref_num_threads())
    out = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "impl": "reference",
           "config": {"workload": {"canyon": WORKLOAD}.get(args.config, WORKLOAD_ARRAY.format(res=RES_APR)),
                      "sample_particles": len(P)},
           "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "reference",
                            "sample": f"{what}; per step, host build of the reference kernels (oracle/_ref)"},
           "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--config", default="array", choices=["canyon", "array", "ensemble", "transfer", "tgv"],
                    help="array: 4x4 cube array with two-level APR, the mixed + learned form against the plain "
                         "FP64 form (default); canyon: the urban-canyon step; "
                         "ensemble: 64 seeded cavity / Taylor-Green cases of 20k-200k particles stepped together; "
                         "transfer: the learned start trained on the canyon's solves, applied to the cube array")
    ap.add_argument("--dx", type=float, default=0.0075, help="transfer config: particle spacing of the cube array")
    ap.add_argument("--train-solves", type=int, default=40, help="transfer config: canyon solves sampled for training")
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--host-control", action="store_true",
                    help="ensemble config: the host-controlled Krylov loop instead of the device-controlled one")
    ap.add_argument("--tol", type=float, default=None, help="PPE tolerance (default 1e-6; tgv config 1e-8)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="precision of the timed form (mixed: FP32 fields and Krylov vectors, FP64 refinement)")
    ap.add_argument("--apr", action=argparse.BooleanOptionalAction, default=True,
                    help="array config: two-level APR near the faces before timing (--no-apr: uniform resolution)")
    ap.add_argument("--mode", default="mixed_ir", choices=["mixed_ir", "bicgstab", "gmres", "idrs", "ref_sweep"])
    ap.add_argument("--fp64-mode", default="bicgstab", choices=["gmres", "bicgstab", "idrs"])
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-cuda", action="store_true",
                    help="skip the reference's own CUDA program (baseline/_ref) on the config's deck")
    ap.add_argument("--no-nnps-check", action="store_true",
                    help="array config: skip the NNPS / neighbour-list comparison with the CPU oracle")
    ap.add_argument("--matrix-free", action="store_true")
    ap.add_argument("--wide-index", action="store_true",
                    help="pressure operator on 32-bit neighbour indices instead of the 16-bit codes")
    ap.add_argument("--coarse", type=int, default=None,
                    help="two-level BiCGSTAB preconditioner: aggregate edge in NNPS cells (0: Jacobi; -B: "
                         "aggregates balanced by row count from blocks of B^3 cells; default 5 for the canyon, -16 "
                         "for the cube array)")
    ap.add_argument("--coarse-max", type=int, default=None,
                    help="balanced coarse space (--coarse < 0): most aggregates (0: 4096, at most 32768; default "
                         "16384)")
    ap.add_argument("--coarse-mode", default="additive", choices=["additive", "multiplicative"],
                    help="two-level form: D^-1 r + Z E^-1 Z^T r, or the coarse correction of the residual the "
                         "Jacobi step leaves (one more operator application per preconditioner call)")
    ap.add_argument("--pair-h", default=None, choices=["ref", "avg"],
                    help="smoothing length of a pair in the pressure system: h_i as the reference's KERNEL_PPE3D "
                         "(ref), or (h_i + h_j)/2, its commented-out multi-resolution form (avg); default avg with "
                         "--apr, else ref")
    ap.add_argument("--gmres-restart", type=int, default=0, help="GMRES(m) restart length (0: 40)")
    ap.add_argument("--inner-tol", type=float, default=0.0, help="restarted refinement: inner tolerance (0: 1e-3)")
    ap.add_argument("--warm", default=None, choices=["prev", "scaled", "extrap", "learned"],
                    help="PPE start vector: previous pressure, previous pressure times its residual-minimising factor, linear "
                         "extrapolation in time, or the learned "
                         "per-particle network (trained on this run's warm-up solves); default learned for the "
                         "array config, previous pressure otherwise")
    ap.add_argument("--pforce-form", default=None, choices=["active", "difference"],
                    help="pressure-force pair term: the reference's active form, or its commented-out difference "
                         "form (no force from a constant pressure); default difference with APR, else active")
    ap.add_argument("--coef-half", action=argparse.BooleanOptionalAction, default=True,
                    help="FP32 operator applications of the mixed form read row-scaled FP16 coefficients "
                         "(ppe_coef_half; default on)")
    ap.add_argument("--start-proj", default="none", choices=["none", "galerkin", "ls"],
                    help="start vector projected on [previous pressure change, coarse correction of the start "
                         "residual, network prediction with --warm learned]: Galerkin or least squares")
    ap.add_argument("--refinement", default="reliable", choices=["reliable", "restart-bicgstab", "restart-gmres",
                                                                  "restart-idrs"],
                    help="mixed_ir form: FP64 reliable updates, or refinement restarting the FP32 solver")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.config == "ensemble":
        return run_ensemble(args, rank, world, local)
    if args.config == "transfer":
        return run_transfer(args, rank, world, local)
    if args.warmup < 3:
        args.warmup = 3
    if args.config != "array":
        args.apr = False
    if args.warm is None:
        args.warm = "learned" if args.config == "array" else "prev"

    import numpy as np
    import torch
    import torch.distributed as dist
    from sph_b200 import abi, decks, layout, replicas

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    boxes = None
    if args.config == "array":
        P, p, boxes = decks.cube_array(scale=args.scale, apr=args.apr)
    elif args.config == "tgv":
        P, p = decks.tgv_periodic(n=int(round(64 * args.scale)))
    else:
        P, p = decks.canyon(scale=args.scale)
    if args.coarse is None:
        args.coarse = {"array": -16, "tgv": 4}.get(args.config, 5)
    if args.coarse_max is None:
        args.coarse_max = 16384 if args.coarse < 0 else 0
    if args.tol is None:
        args.tol = 1e-8 if args.config == "tgv" else 1e-6
    mode = {"mixed_ir": layout.PPE_MIXED_IR, "bicgstab": layout.PPE_BICGSTAB, "gmres": layout.PPE_GMRES,
            "idrs": layout.PPE_IDRS, "ref_sweep": layout.PPE_REF_SWEEP}[args.mode]
    p.ppe_mode = mode
    p.ppe_tol = args.tol
    if args.matrix_free:
        p.ppe_matrix_free = 1
    p.ppe_wide_index = 1 if args.wide_index else 0
    p.ppe_coef_half = 1 if args.coef_half else 0
    p.ppe_refinement = {"reliable": 0, "restart-gmres": 1, "restart-bicgstab": 2, "restart-idrs": 3}[args.refinement]
    p.ppe_coarse_block = args.coarse
    p.ppe_coarse_max = args.coarse_max
    p.ppe_coarse_mode = 1 if args.coarse_mode == "multiplicative" else 0
    if args.pair_h is None:
        args.pair_h = "avg" if args.apr else "ref"
    p.ppe_pair_h = 1 if args.pair_h == "avg" else 0
    if args.pforce_form is None:
        args.pforce_form = "difference" if args.apr else "active"
    p.pressure_force_form = 1 if args.pforce_form == "difference" else 0
    p.ppe_gmres_restart = args.gmres_restart
    if args.inner_tol > 0:
        p.ppe_inner_tol = args.inner_tol
    p.ppe_warm_start = {"extrap": 1, "scaled": 3}.get(args.warm, 0)
    if args.start_proj != "none":
        p.ppe_warm_start = 4 if args.start_proj == "galerkin" else 5
    # particle-steps count particles, not the periodic ghost records
    n = int((P["buffer_type"] != layout.BUFFER_PERIODIC_GHOST).sum())
    prec = layout.PREC_FP64 if args.precision == "fp64" else layout.PREC_MIXED
    # the context's own stream: the Krylov iterations between host checks
    # replay as a CUDA graph (the legacy default stream cannot be captured)
    stream = torch.cuda.Stream(device=local)
    sim = abi.Simulation(p, precision=prec, device=local, stream=ctypes.c_void_p(stream.cuda_stream))
    if boxes is not None:
        sim.set_ib_boxes(boxes)
    sim.upload(P)
    apr = None
    if args.config == "array" and args.apr:
        # two-level APR near the faces before timing: splitting passes until no
        # cell asks (one particle per cell and pass); every form starts from
        # the refined state
        passes, split = 0, 0
        for passes in range(1, 16):
            ns, _ = sim.apr()
            split += ns
            if ns == 0:
                break
        P, _, _ = sim.download()
        n = int((P["i_type"] < 3).sum())   # particle-steps count active particles, not free records
        apr = {"passes": passes, "cells_split": split, "active_particles": n, "records": len(P)}
    # the first step builds what the later ones reuse (neighbour lists, the
    # stored pair factors and coefficients, the coarse space and its inverse)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.step(1)
    torch.cuda.synchronize()
    first_step_s = time.perf_counter() - t0
    learned = None
    if args.warm == "learned":
        # samples from the warm-up solves, then Adam on the GPU (not timed)
        every = max(1, n // 250000)
        sim.ml_collect(every)
        wsteps = max(args.warmup, 8)
        for _ in range(wsteps):
            sim.step(1)
        sim.ml_collect(0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss = sim.ml_train(epochs=6, batch=4096, lr=1e-3, seed=20261203)
        train_s = time.perf_counter() - t0
        nsamp = int(lib_sample_count(sim))
        q = p.copy()
        q.ppe_mode = layout.PPE_LEARNED
        sim.set_params(q)
        learned = {"samples": nsamp, "warmup_steps_collected": wsteps, "every_kth_fluid_row": every,
                   "train_s": train_s, "train_loss": loss, "epochs": 6, "batch": 4096}
        for _ in range(2):
            sim.step(1)
        ml_weights = sim.ml_get_weights()
    else:
        ml_weights = None
        for _ in range(args.warmup):
            sim.step(1)

    # ---- device-timed region ----
    clocks = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sim.profile(True)
    sim.operator_stats(reset=True)
    l0 = sim.launches()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stats, phases = [], []
    e0.record(stream)
    for _ in range(args.steps):
        s = sim.step(1)
        stats.append((s.iterations, s.refinements, s.rel_residual, s.solve_ms, s.status, s.initial_residual))
        phases.append(sim.phase_ms().copy())
    e1.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = sim.launches() - l0
    op_n, op_ms, op_bytes = sim.operator_stats(reset=True)
    op_counts = sim.operator_counts()
    _, op_index_bytes = sim.operator_bytes()
    sim.profile(False)
    value, ms = replicas.throughput(n, args.steps, ms, device="cuda")

    # ---- end to end through the C ABI with host buffers ----
    host = torch.empty(len(P) * layout.PART1.itemsize, dtype=torch.uint8, pin_memory=True).numpy().view(layout.PART1)
    sim.download_into(host)
    ke = max(3, args.steps // 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    seg = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(ke)]
    for k in range(ke):
        sim.upload_state(host)
        seg[k][0].record(stream)
        sim.step(1)
        seg[k][1].record(stream)
        sim.download_into(host)
        seg[k][2].record(stream)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    # where the end-to-end time goes: upload (H2D + unpack), step, download (pack + D2H)
    e2e_split = {"upload_ms": (f0.elapsed_time(seg[0][0])
                               + sum(seg[k - 1][2].elapsed_time(seg[k][0]) for k in range(1, ke))) / ke,
                 "step_ms": sum(seg[k][0].elapsed_time(seg[k][1]) for k in range(ke)) / ke,
                 "download_ms": sum(seg[k][1].elapsed_time(seg[k][2]) for k in range(ke)) / ke}
    e2e, e2e_ms = replicas.throughput(n, ke, e2e_ms, device="cuda")

    # ---- other forms on the same deck, rank 0 only ----
    sim.close()

    def timed_form(precision, mode, coarse, steps, keep=False, weights=None):
        q = p.copy()
        q.ppe_mode = mode
        q.ppe_coarse_block = coarse
        sd = abi.Simulation(q, precision=precision, device=local)
        if boxes is not None:
            sd.set_ib_boxes(boxes)
        if weights is not None:
            sd.ml_set_weights(weights)
        sd.upload(P)
        for _ in range(2):
            sd.step(1)
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        dstats = []
        g0.record()
        for _ in range(steps):
            s = sd.step(1)
            dstats.append((s.iterations, s.rel_residual, s.solve_ms))
        g1.record()
        torch.cuda.synchronize()
        dms = g0.elapsed_time(g1)
        state = sd.download(want=(1,))[0] if keep else None
        sd.close()
        out = {"value": n * steps / (dms / 1e3), "ms_per_step": dms / steps, "steps": steps,
               "ppe_ms": statistics.mean(d[2] for d in dstats),
               "ppe_iterations": statistics.mean(d[0] for d in dstats),
               "rel_residual_max": max(d[1] for d in dstats)}
        if keep:
            out["_state"] = state
        return out

    def error_vs(ref_state, steps):
        """The chosen form run from the same start for the same number of
        steps as the FP64 form, and its relative error against it over the
        fluid particles (form_error)."""
        if ref_state is None:
            return None
        q = p.copy()
        if ml_weights is not None:   # the learned form with this run's trained network
            q.ppe_mode = layout.PPE_LEARNED
        sd = abi.Simulation(q, precision=layout.PREC_MIXED, device=local)
        if boxes is not None:
            sd.set_ib_boxes(boxes)
        if ml_weights is not None:
            sd.ml_set_weights(ml_weights)
        sd.upload(P)
        for _ in range(steps):
            sd.step(1)
        A = sd.download(want=(1,))[0]
        sd.close()
        out = {"steps": steps}
        out.update(form_error(A, ref_state, p.getf("u_limit")))
        return out

    fp64 = fp64_same = sweep = err64 = learned_vs_prev = None
    if rank == 0:
        kd = max(3, args.steps // 4)
        fp64_mode = layout.PPE_GMRES if args.fp64_mode == "gmres" else layout.PPE_BICGSTAB
        if not args.no_fp64:
            # the plain form: FP64 throughout, Jacobi-preconditioned Krylov
            fp64 = timed_form(layout.PREC_FP64, fp64_mode, 0, kd, keep=True)
            fp64.update({"solver": args.fp64_mode + " + jacobi", "ppe_tol": args.tol})
            err64 = error_vs(fp64.pop("_state"), kd + 2)
            if args.coarse != 0:
                # FP64 with this run's preconditioner: isolates the precision change
                fp64_same = timed_form(layout.PREC_FP64, layout.PPE_BICGSTAB, args.coarse, kd)
                fp64_same.update({"solver": f"bicgstab + coarse {args.coarse}", "ppe_tol": args.tol})
        if ml_weights is not None:
            # the learned start against the previous pressure, same start, same steps
            prev_same = timed_form(layout.PREC_MIXED, layout.PPE_MIXED_IR, args.coarse, kd)
            learned_same = timed_form(layout.PREC_MIXED, layout.PPE_LEARNED, args.coarse, kd, weights=ml_weights)
            learned_vs_prev = {"steps": kd, "previous_pressure": prev_same, "learned": learned_same,
                               "iterations_saved_per_step": prev_same["ppe_iterations"] -
                               learned_same["ppe_iterations"],
                               "ms_saved_per_step": prev_same["ms_per_step"] - learned_same["ms_per_step"]}
        # the reference's own step semantics (one PPE sweep) on the same deck
        sweep = timed_form(layout.PREC_MIXED, layout.PPE_REF_SWEEP, 0, kd)
        for k in ("ppe_iterations", "rel_residual_max"):
            sweep.pop(k)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0

    hbm, peak_kind = peaks()
    per_launch_ms = op_ms / max(op_n, 1)
    # the roofline counts per-row fields and 4 B per stored neighbour index
    # (sph_operator_bytes' index rule); the stored-layout figure (cached
    # coefficients and 16-bit codes streamed per launch) is reported beside it
    achieved = op_index_bytes / (per_launch_ms / 1e3) / 1e9 if op_n else 0.0
    achieved_stored = op_bytes / (per_launch_ms / 1e3) / 1e9 if op_n else 0.0
    # DRAM bytes per launch from the committed ncu capture of this config's
    # operator on a smaller deck, scaled by the stored bytes of a launch
    # (rows, stored entries and Neumann entries grow together)
    nc = ncu_traffic(f"ppe_operator_{args.config}.json")
    traffic = None
    if (nc and "measured_at" in nc and nc.get("apr", False) == bool(args.apr)
            and nc.get("coef_half", False) == bool(p.ppe_coef_half)
            and nc.get("entries_counted") == "fluid rows"):
        m = nc["measured_at"]
        traffic = m["traffic_over_algorithmic"] * op_bytes
    ph = np.mean(np.array(phases), axis=0) if phases else np.zeros(4)
    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64",
        "data": "synthetic",
        "config": {"workload": {"canyon": WORKLOAD,
                                "array": WORKLOAD_ARRAY.format(res=RES_APR if args.apr else RES_UNIFORM)}.get(
                       args.config, WORKLOAD_TGV.format(n=int(round(64 * args.scale)))),
                   "particles": n, "apr": apr, "scale": args.scale,
                   "precision": "mixed FP32/FP64" if args.precision == "mixed" else "FP64",
                   "ppe": args.mode, "ppe_tol": args.tol,
                   "ppe_operator": "matrix-free" if args.matrix_free else
                   ("cached c_ij, 16-bit neighbour codes" if op_counts["codes16"] else
                    "cached c_ij, 32-bit neighbour indices" + ("" if args.wide_index else
                                                               " (16-bit codes asked for, not representable)"))
                   + (", FP16 row-scaled c_ij in the FP32 applications" if args.coef_half else ""),
                   "ppe_refinement": args.refinement,
                   "ppe_pair_h": {"ref": "h_i", "avg": "(h_i + h_j) / 2"}[args.pair_h],
                   "ppe_start_projection": args.start_proj,
                   "pressure_force": {"active": "the reference's active pair term (Monaghan variation)",
                                      "difference": "the reference's commented-out difference form "
                                                    "-m_j (p_j - p_i) / (rho_i rho_j)"}[args.pforce_form],
                   "ppe_start_vector": {"prev": "previous pressure", "extrap": "linear extrapolation in time",
                                        "scaled": "previous pressure times its residual-minimising factor",
                                        "learned": "learned per-particle MLP on the previous pressure"}[args.warm],
                   "ppe_preconditioner": (f"jacobi + coarse aggregates of {args.coarse}^3 cells ({args.coarse_mode})"
                                          if args.coarse > 0 else
                                          f"jacobi + coarse aggregates balanced by row count, octree boxes from "
                                          f"{-args.coarse}^3 cells, at most {args.coarse_max or 4096} "
                                          f"({args.coarse_mode})"
                                          if args.coarse < 0 else "jacobi"),
                   "first_step_s": first_step_s,
                   "l2": "inputs larger than L2 (particle state and neighbour lists exceed 126 MB)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "e2e": {"value": e2e, "unit": METRIC, "split": e2e_split, "h2d_bytes_per_step": len(P) * layout.PART1.itemsize,
                "d2h_bytes_per_step": len(P) * layout.PART1.itemsize, "steps": ke},
        "gpu_launches": int(launches),
        "ppe": {"iterations_mean": statistics.mean(s[0] for s in stats),
                "refinements_mean": statistics.mean(s[1] for s in stats),
                "rel_residual_max": max(s[2] for s in stats),
                "solve_ms_mean": statistics.mean(s[3] for s in stats),
                "initial_residual_mean": statistics.mean(s[5] for s in stats),
                "not_converged_steps": sum(1 for s in stats if s[4] != 0)},
        "phase_ms": {"interaction": float(ph[1]), "ppe": float(ph[2]), "time_update": float(ph[3])},
        "roofline": {"bound": "hbm", "kernel": "PPE operator (k_spmv_fused: SELL rows + Neumann rows, cached c_ij)" if not args.matrix_free
                     else "PPE operator (k_spmv_mf)",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": op_index_bytes,
                     "bytes_rule": "per row its fields read and written, per stored neighbour its 4-byte index",
                     "stored_layout": {"bytes_per_launch": op_bytes, "achieved": achieved_stored,
                                       "frac": achieved_stored / hbm,
                                       "rule": "what the launch streams: 16-bit codes or 32-bit indices plus the "
                                               "cached coefficient per entry, Neumann weights, code tables"},
                     "launch_ms": per_launch_ms, "launches": op_n, "operator_counts": op_counts},
        "plain_fp64": fp64,
        "error_vs_plain_fp64": err64,
        "fp64_same_preconditioner": fp64_same,
        "learned_warm_start": learned,
        "learned_vs_previous_pressure": learned_vs_prev,
        "reference_step_semantics": sweep,
        "clocks": ck,
    }
    if fp64:
        out["mixed_vs_fp64"] = value / fp64["value"] if fp64["value"] else None
    if args.config == "array" and not args.no_nnps_check:
        out["nnps_bit_exact"] = nnps_check(P, p, boxes, local)
    if world == 1 and not args.no_ref_cuda and args.config in ("array", "canyon"):
        out["ref_cuda_baseline"] = ref_cuda_baseline(args.config, 2, 5)
    if world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline_tgv(steps=4) if args.config == "tgv" else cpu_baseline(4, args.config)
        if args.config == "array":
            out["cpu_converged_port"] = cpu_converged_port(local, pforce_form=p.pressure_force_form)
    print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
