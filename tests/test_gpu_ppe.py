"""Converged pressure solves on the GPU (needs a B200).

The reference runs one pressure sweep per step; the converged modes are new
work and are judged against the CPU oracle's FP64 BiCGSTAB on the same
operator (same rows, same pinned rows):
  * FP64 BiCGSTAB: ||b-Ap||/||b|| <= 1e-8 and pressure within PRES_TOL_FP64 of
    the oracle's converged pressure (both solves stop at 1e-8 / 1e-10);
  * mixed form (FP32 BiCGSTAB with FP64 reliable updates): ||b-Ap||/||b||
    <= 1e-6 and velocity within MIXED_TOL of the plain FP64 form solved to
    1e-9; pressure within MIXED_PRES_TOL, because a 1e-6 residual bounds the
    pressure error only through the conditioning of the Poisson operator
    (smooth error modes), which the velocity update sees through a gradient;
  * the matrix-free operator gives the cached operator's answer.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

import restated

pytestmark = pytest.mark.gpu

PRES_TOL_FP64 = 1e-6
MIXED_TOL = 1e-4
MIXED_PRES_TOL = 1e-3


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _gpu_step(P, p, precision, mode, tol, nsteps=1, matrix_free=False, coarse=0, coef_half=0):
    q = p.copy()
    q.ppe_coef_half = coef_half
    q.ppe_mode = mode
    q.ppe_tol = tol
    q.ppe_max_iter = 4000
    q.ppe_coarse_block = coarse
    if matrix_free:
        q.ppe_matrix_free = 1
    sim = abi.Simulation(q, precision=precision)
    sim.upload(P)
    stats = [sim.step(1) for _ in range(nsteps)]
    A, _, _ = sim.download()
    sim.close()
    return A, stats


@pytest.fixture(scope="module")
def deck():
    return decks.caseh_mini(nx=14, ny=8, nz=5)


def test_fp64_bicgstab_matches_oracle(deck):
    P, p = deck
    A, stats = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-8)
    assert stats[-1].status == 0 and stats[-1].rel_residual <= 1e-8, (stats[-1].rel_residual, stats[-1].iterations)
    O = restated.Restated(P, p, 1)
    st, rel, it = O.step(1, mode=layout.PPE_BICGSTAB, tol=1e-10, maxit=5000)
    assert st == 0
    B, _, _ = O.download()
    assert rel_err(A["pres"], B["pres"]) <= PRES_TOL_FP64
    for f in ("ux", "uy", "uz"):
        assert rel_err(A[f], B[f]) <= PRES_TOL_FP64, f


def test_mixed_ir_reaches_tolerance_and_matches_fp64(deck):
    P, p = deck
    A, st32 = _gpu_step(P, p, layout.PREC_MIXED, layout.PPE_MIXED_IR, 1e-6, nsteps=2)
    for s in st32:
        assert s.status == 0 and s.rel_residual <= 1e-6, (s.rel_residual, s.iterations, s.refinements)
    B, st64 = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_GMRES, 1e-9, nsteps=2)
    assert rel_err(A["pres"], B["pres"]) <= MIXED_PRES_TOL
    for f in ("ux", "uy", "uz"):
        assert rel_err(A[f], B[f]) <= MIXED_TOL, f


def test_fp32_gmres_converges(deck):
    P, p = deck
    A, st = _gpu_step(P, p, layout.PREC_MIXED, layout.PPE_GMRES, 1e-5, nsteps=2)
    for s in st:
        assert s.status == 0 and s.rel_residual <= 1e-5


def test_fp64_gmres_matches_oracle(deck):
    P, p = deck
    A, stats = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_GMRES, 1e-9)
    assert stats[-1].status == 0 and stats[-1].rel_residual <= 1e-9
    O = restated.Restated(P, p, 1)
    st, rel, it = O.step(1, mode=layout.PPE_BICGSTAB, tol=1e-10, maxit=5000)
    assert st == 0
    B, _, _ = O.download()
    assert rel_err(A["pres"], B["pres"]) <= PRES_TOL_FP64


def test_matrix_free_equals_cached(deck):
    P, p = deck
    A, s1 = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-9)
    B, s2 = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-9, matrix_free=True)
    assert s1[-1].status == 0 and s2[-1].status == 0
    assert rel_err(A["pres"], B["pres"]) <= 1e-7


def test_not_converged_status_with_tiny_iteration_budget(deck):
    P, p = deck
    q = p.copy()
    q.ppe_mode = layout.PPE_BICGSTAB
    q.ppe_tol = 1e-12
    q.ppe_max_iter = 3
    sim = abi.Simulation(q, precision=layout.PREC_FP64)
    sim.upload(P)
    s = sim.step(1)
    assert s.status == 1 and s.iterations <= 3
    sim.close()


def test_fp64_coarse_preconditioner_matches_oracle_in_fewer_iterations(deck):
    # Jacobi + coarse aggregates of 2^3 cells against Jacobi alone: the same
    # converged pressure (the operator is unchanged) in fewer iterations
    P, p = deck
    A0, s0 = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-8)
    A1, s1 = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-8, coarse=2)
    assert s1[-1].status == 0 and s1[-1].rel_residual <= 1e-8
    assert s1[-1].iterations < s0[-1].iterations, (s1[-1].iterations, s0[-1].iterations)
    O = restated.Restated(P, p, 1)
    st, rel, it = O.step(1, mode=layout.PPE_BICGSTAB, tol=1e-10, maxit=5000)
    assert st == 0
    B, _, _ = O.download()
    assert rel_err(A1["pres"], B["pres"]) <= PRES_TOL_FP64
    for f in ("ux", "uy", "uz"):
        assert rel_err(A1[f], B[f]) <= PRES_TOL_FP64, f


def test_mixed_coarse_reaches_tolerance_and_matches_fp64(deck):
    P, p = deck
    A, st32 = _gpu_step(P, p, layout.PREC_MIXED, layout.PPE_MIXED_IR, 1e-6, nsteps=2, coarse=2)
    for s in st32:
        assert s.status == 0 and s.rel_residual <= 1e-6, (s.rel_residual, s.iterations, s.refinements)
    B, _ = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_GMRES, 1e-9, nsteps=2)
    assert rel_err(A["pres"], B["pres"]) <= MIXED_PRES_TOL
    for f in ("ux", "uy", "uz"):
        assert rel_err(A[f], B[f]) <= MIXED_TOL, f


@pytest.mark.parametrize("coarse", [0, 2], ids=["jacobi", "two_level"])
def test_fp16_coefficients_reach_tolerance_and_match_fp64(deck, coarse):
    """ppe_coef_half: the FP32 applications read FP16 row-scaled c_ij; the
    FP64 true residuals keep the FP32 coefficients, so the solve still ends
    at ||b - Ap|| <= 1e-6 ||b|| and the step stays within the mixed form's bar."""
    P, p = deck
    A, st = _gpu_step(P, p, layout.PREC_MIXED, layout.PPE_MIXED_IR, 1e-6, nsteps=2, coarse=coarse, coef_half=1)
    for s in st:
        assert s.status == 0 and s.rel_residual <= 1e-6, (s.rel_residual, s.iterations, s.refinements)
    B, _ = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_GMRES, 1e-9, nsteps=2)
    assert rel_err(A["pres"], B["pres"]) <= MIXED_PRES_TOL
    for f in ("ux", "uy", "uz"):
        assert rel_err(A[f], B[f]) <= MIXED_TOL, f


def test_coarse_block_too_small_is_rejected(deck):
    # one aggregate per cell exceeds the aggregate limit on a deck with more
    # than 16384 occupied cells: the solve reports SPH_ERR_UNSUPPORTED
    P, p = decks.canyon(scale=1.0)
    q = p.copy()
    q.ppe_mode = layout.PPE_BICGSTAB
    q.ppe_coarse_block = 1
    sim = abi.Simulation(q, precision=layout.PREC_MIXED)
    sim.upload(P)
    with pytest.raises(abi.SphError) as e:
        sim.step(1)
    assert e.value.status == -7
    sim.close()


def test_balanced_coarse_space_converges_in_fewer_iterations():
    # aggregates balanced by row count (ppe_coarse_block = -B) up to
    # ppe_coarse_max: with the blocked Gauss-Jordan inverse (checked on four
    # of its columns inside the build) the FP64 solve reaches the pressure of
    # the Jacobi-only solve (both to 1e-8) in fewer iterations, and more
    # aggregates need fewer iterations
    P, p = decks.canyon(scale=0.3)
    A0, s0 = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-8)
    assert s0[-1].status == 0
    iters = {}
    for cmax in (4096, 12000):
        q = p.copy()
        q.ppe_coarse_max = cmax
        A1, s1 = _gpu_step(P, q, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-8, coarse=-4)
        assert s1[-1].status == 0 and s1[-1].rel_residual <= 1e-8
        assert rel_err(A1["pres"], A0["pres"]) <= PRES_TOL_FP64
        for f in ("ux", "uy", "uz"):
            assert rel_err(A1[f], A0[f]) <= PRES_TOL_FP64, f
        iters[cmax] = s1[-1].iterations
    assert iters[12000] < iters[4096] < s0[-1].iterations, (iters, s0[-1].iterations)


def _two_level_deck():
    """caseh_mini with the smoothing length of the channel's downstream half
    (0.3 m < x, before the outlet block at L3) raised by half, so that pairs
    across the level interface have h_i != h_j."""
    P, p = decks.caseh_mini(nx=14, ny=8, nz=5)
    P = P.copy()
    far = (P["x"] > np.float32(0.3)) & (P["x"] < np.float32(5.0))
    P["h"][far] *= np.float32(1.5)
    P["h_ref"][far] = P["h"][far]
    decks.domain_setup(p, P)
    return P, p


def test_pair_averaged_h_matches_oracle():
    """ppe_pair_h = 1 (the reference's commented-out multi-resolution form of
    the pressure rows): FP64 BiCGSTAB against the oracle with the same
    option, the matrix-free operator against the cached one, and a pressure
    different from the h_i form on a deck with two smoothing lengths."""
    P, p = _two_level_deck()
    q = p.copy()
    q.ppe_pair_h = 1
    A, stats = _gpu_step(P, q, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-8)
    assert stats[-1].status == 0 and stats[-1].rel_residual <= 1e-8
    O = restated.Restated(P, q, 1)
    st, rel, it = O.step(1, mode=layout.PPE_BICGSTAB, tol=1e-10, maxit=5000)
    assert st == 0
    B, _, _ = O.download()
    assert rel_err(A["pres"], B["pres"]) <= PRES_TOL_FP64
    M, s2 = _gpu_step(P, q, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-8, matrix_free=True)
    assert s2[-1].status == 0 and rel_err(M["pres"], A["pres"]) <= 1e-6
    R, s3 = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-8)
    assert s3[-1].status == 0 and rel_err(R["pres"], A["pres"]) > 1e-4


def test_fp64_idrs_matches_oracle(deck):
    """IDR(4) in the FP64 form (with the two-level preconditioner) converges
    to the oracle's FP64 BiCGSTAB pressure."""
    P, p = deck
    A, stats = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_IDRS, 1e-8, coarse=2)
    assert stats[-1].status == 0 and stats[-1].rel_residual <= 1e-8, (stats[-1].rel_residual, stats[-1].iterations)
    O = restated.Restated(P, p, 1)
    st, rel, it = O.step(1, mode=layout.PPE_BICGSTAB, tol=1e-10, maxit=5000)
    assert st == 0
    B, _, _ = O.download()
    assert rel_err(A["pres"], B["pres"]) <= PRES_TOL_FP64


def test_mixed_refinement_with_idrs_matches_fp64(deck):
    """Refinement restarting FP32 IDR(4) (ppe_refinement = 3) reaches the
    tolerance and the velocity of the FP64 form."""
    P, p = deck
    q = p.copy()
    q.ppe_refinement = 3
    A, s1 = _gpu_step(P, q, layout.PREC_MIXED, layout.PPE_MIXED_IR, 1e-6, coarse=2)
    B, s2 = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-9, coarse=2)
    assert s1[-1].status == 0 and s1[-1].rel_residual <= 1e-6
    for f in ("ux", "uy", "uz"):
        assert rel_err(A[f], B[f]) <= MIXED_TOL, f


def _tgv_amplitude(A):
    it = A["buffer_type"] != layout.BUFFER_PERIODIC_GHOST
    k = 2 * np.pi
    x, y, z = (A[c][it].astype(np.float64) for c in "xyz")
    ua = np.sin(k * x) * np.cos(k * y) * np.cos(k * z)
    return float((A["ux"][it] * ua).sum() / (ua * ua).sum())


@pytest.mark.parametrize("coarse", [0, 2], ids=["jacobi", "two_level"])
def test_tgv_fp64_bicgstab_matches_oracle(coarse):
    """Triply periodic box (ghost rows are copy rows, the operator is
    singular): the FP64 solve matches the oracle's pressure and velocity."""
    P, p = decks.tgv_periodic(n=12)
    A, stats = _gpu_step(P, p, layout.PREC_FP64, layout.PPE_BICGSTAB, 1e-8, nsteps=2, coarse=coarse)
    for s in stats:
        assert s.status == 0 and s.rel_residual <= 1e-8, (s.rel_residual, s.iterations)
    O = restated.Restated(P, p, 1)
    for _ in range(2):
        st, rel, it = O.step(1, mode=layout.PPE_BICGSTAB, tol=1e-10, maxit=5000)
        assert st == 0
    B, _, _ = O.download()
    assert rel_err(A["pres"], B["pres"]) <= PRES_TOL_FP64
    for f in ("ux", "uy", "uz"):
        assert rel_err(A[f], B[f]) <= PRES_TOL_FP64, f


def test_tgv_mixed_decay_rate():
    """The mixed form on the Taylor-Green box decays as exp(-3 nu k^2 t)
    (Re = 20, 16^3 lattice, 20 steps) like the oracle's FP64 step."""
    P, p = decks.tgv_periodic(n=16, nu=0.05)
    A, stats = _gpu_step(P, p, layout.PREC_MIXED, layout.PPE_BICGSTAB, 1e-6, nsteps=20, coarse=2)
    assert all(s.status == 0 for s in stats)
    t = 20 * p.getf("dt")
    want = np.exp(-3 * 0.05 * (2 * np.pi) ** 2 * t)
    assert abs(_tgv_amplitude(A) / want - 1) < 1e-2


def test_graph_replay_with_live_timing_matches_stream_launches(deck):
    """Contexts on their own stream replay the mixed BiCGSTAB iterations as a
    CUDA graph; with live operator timing on, the graph carries event nodes
    around each operator application.  Both give exactly the results of the
    same steps launched one kernel at a time on the legacy stream, and the
    timed graph reports every operator application."""
    import ctypes

    import torch
    P, p = deck
    q = p.copy()
    q.ppe_mode = layout.PPE_MIXED_IR
    q.ppe_tol = 1e-6
    q.ppe_coarse_block = 2
    out = []
    for own, prof in ((False, False), (True, False), (True, True)):
        s = torch.cuda.Stream() if own else None
        sim = abi.Simulation(q, precision=layout.PREC_MIXED, stream=ctypes.c_void_p(s.cuda_stream) if own else None)
        sim.upload(P)
        sim.profile(prof)
        sim.operator_stats(reset=True)
        st = [sim.step(1) for _ in range(3)]
        n_op, ms, _ = sim.operator_stats(reset=True)
        A, _, _ = sim.download()
        sim.close()
        assert all(x.status == 0 for x in st)
        out.append((A, st, n_op, ms))
    for f in ("ux", "uy", "uz", "pres"):
        assert np.array_equal(out[0][0][f], out[1][0][f]), f
        assert np.array_equal(out[0][0][f], out[2][0][f]), f
    its = sum(x.iterations for x in out[2][1])
    # two timed applications per iteration (graph chunks run whole chunks of
    # four, the solve stops counting at convergence)
    assert out[2][2] >= 2 * its and out[2][3] > 0


@pytest.mark.parametrize("name", ["caseh_mini", "tgv_periodic", "canyon_small"])
def test_16bit_neighbour_codes_give_identical_steps(name):
    """The pressure operator reading 16-bit neighbour codes (default) visits
    the same entries in the same order as with 32-bit indices
    (ppe_wide_index = 1): the mixed and FP64 steps are bit-identical, and the
    operator's algorithmic bytes show which form ran."""
    P, p = {"caseh_mini": lambda: decks.caseh_mini(nx=14, ny=8, nz=5),
            "tgv_periodic": lambda: decks.tgv_periodic(n=10),
            "canyon_small": lambda: decks.canyon(scale=0.12)}[name]()
    for precision in (layout.PREC_MIXED, layout.PREC_FP64):
        out = []
        for wide in (0, 1):
            q = p.copy()
            q.ppe_mode = layout.PPE_MIXED_IR
            q.ppe_tol = 1e-6
            q.ppe_coarse_block = 2
            q.ppe_wide_index = wide
            sim = abi.Simulation(q, precision=precision)
            sim.upload(P)
            st = [sim.step(1) for _ in range(2)]
            _, _, nbytes = sim.operator_stats(reset=True)
            A, _, _ = sim.download()
            sim.close()
            assert all(s.status == 0 for s in st)
            out.append((A, [s.iterations for s in st], nbytes))
        assert out[0][2] < out[1][2]
        assert out[0][1] == out[1][1]
        for f in ("ux", "uy", "uz", "pres"):
            assert np.array_equal(out[0][0][f], out[1][0][f]), (precision, f)
