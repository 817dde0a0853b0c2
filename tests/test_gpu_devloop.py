"""The mixed form's solve under device control (ppe_refinement = 4), needs a
B200.

The whole solve is one CUDA graph whose conditional nodes take the host
loop's decisions (reliable updates, restarts, convergence), so it must give
the host-controlled solve's iterates exactly: the same pressure and velocity
bit for bit and the same iteration and update counts, over several steps
stepped in one sph_step call (whose statistics the host reads once, at the
end), also when later steps replay the whole step as one captured graph.  A budget too small to converge must come back as SPH_NOT_CONVERGED,
and an ensemble of cases under device control must equal its cases stepped
alone.
"""
import ctypes

import numpy as np
import pytest

from sph_b200 import abi, decks, layout

pytestmark = pytest.mark.gpu


def _run(P, p, refinement, steps, per_call=1, max_iter=2000, coarse=2, calls=None):
    import torch
    q = p.copy()
    q.ppe_mode = layout.PPE_MIXED_IR
    q.ppe_tol = 1e-6
    q.ppe_coarse_block = coarse
    q.ppe_refinement = refinement
    q.ppe_max_iter = max_iter
    stream = torch.cuda.Stream(device=0)
    sim = abi.Simulation(q, precision=layout.PREC_MIXED, stream=ctypes.c_void_p(stream.cuda_stream))
    sim.upload(P)
    stats = []
    status = []
    for k in (calls or [per_call] * (steps // per_call)):
        try:
            stats.append(sim.step(k))
            status.append(0)
        except abi.SphError as e:
            status.append(e.status)
            break
    A, _, _ = sim.download()
    _run.graph_steps = sim.graph_steps()
    sim.close()
    return A, stats, status


@pytest.mark.parametrize("coarse", [0, 2], ids=["jacobi", "two_level"])
def test_device_controlled_solve_equals_host_loop(coarse):
    P, p = decks.canyon(scale=0.12)
    A, sa, _ = _run(P, p, 0, 3, coarse=coarse)
    B, sb, _ = _run(P, p, 4, 3, coarse=coarse)
    for f in ("pres", "ux", "uy", "uz"):
        assert np.array_equal(A[f], B[f]), f
    for x, y in zip(sa, sb):
        assert (x.iterations, x.refinements, x.restarts, x.status) == (y.iterations, y.refinements, y.restarts, y.status)
        assert x.rel_residual == pytest.approx(y.rel_residual, rel=1e-12)
        assert x.rel_residual <= 1e-6


def test_device_controlled_steps_in_one_call():
    P, p = decks.canyon(scale=0.12)
    A, sa, _ = _run(P, p, 0, 4, per_call=1)
    assert _run.graph_steps == 0
    B, sb, _ = _run(P, p, 4, 4, per_call=4)     # four steps, statistics read once
    # steps 0 and 1 launch by launch, step 2 captured as one graph, 2 and 3
    # replays of it
    assert _run.graph_steps == 2
    for f in ("pres", "ux", "uy", "uz"):
        assert np.array_equal(A[f], B[f]), f
    last = sb[-1]
    assert (last.iterations, last.refinements) == (sa[-1].iterations, sa[-1].refinements)
    assert last.rel_residual <= 1e-6 and last.solve_ms > 0


def test_device_controlled_budget_reports_not_converged():
    P, p = decks.canyon(scale=0.12)
    _, sa, _ = _run(P, p, 0, 1, max_iter=8)
    _, sb, _ = _run(P, p, 4, 1, max_iter=8)
    assert sa[0].status == 1 and sb[0].status == 1     # SPH_NOT_CONVERGED
    assert sa[0].iterations == sb[0].iterations


def test_whole_step_graph_follows_the_step_counter():
    # a filter period of 2 and a wall-temperature ramp over the first steps
    # (the time update sets the walls' temperature from the step's time): the
    # replayed graph reads the step counter and time from the device, so it
    # must give the launch-by-launch results at every step, also across
    # sph_step calls
    P, p = decks.canyon(scale=0.12)
    p.seti("freq_filt", 2)
    dt = p.getf("dt")
    p.t_ini, p.t_con, p.t_start, p.t_con_t = 300.0, 304.0, dt, 6.0 * dt
    A, sa, ra = _run(P, p, 0, 7, per_call=1)
    B, sb, rb = _run(P, p, 4, 7, calls=[5, 2])
    assert ra == [0] * 7 and rb == [0, 0]   # every solve converged
    assert _run.graph_steps == 5       # steps 2-6
    for f in ("pres", "ux", "uy", "uz", "temp"):
        assert np.array_equal(A[f], B[f]), f
    assert (sa[-1].iterations, sa[-1].refinements) == (sb[-1].iterations, sb[-1].refinements)
