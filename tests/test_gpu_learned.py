"""Learned warm start of the pressure solve on the GPU (needs a B200).

* gradients of the FP32 training kernels against the CPU restatement
  (oracle/mlp.py, FP64) on samples the solver itself collected;
* tensor-core (BF16) inference against the restatement's bit-exact emulation
  of its BF16 rounding;
* what the trained network gains: the same deck stepped from the same state
  with and without the warm start.  The network's start vector has a lower
  residual than the previous pressure (the quantity it is trained and scaled
  for); both solves reach 1e-6 and the two velocity fields agree to 1e-4.
  The Krylov iteration counts of both are recorded, not asserted: on this
  operator a lower start residual has not meant fewer BiCGSTAB iterations.
"""
import numpy as np
import pytest

from sph_b200 import abi, decks, layout

import mlp

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4      # relative 2-norm error of the FP32 gradient vs FP64
INFER_TOL = 2e-3     # relative 2-norm error of the BF16 inference vs its emulation


def _collecting_sim(steps=3, every=1, coarse=2, scale=0.12):
    P, p = decks.canyon(scale=scale)
    q = p.copy()
    q.ppe_mode = layout.PPE_MIXED_IR
    q.ppe_tol = 1e-6
    q.ppe_coarse_block = coarse
    sim = abi.Simulation(q, precision=layout.PREC_MIXED)
    sim.upload(P)
    sim.ml_collect(every)
    for _ in range(steps):
        s = sim.step(1)
        assert s.status == 0
    return sim, P, q


def _features(X):
    return mlp.bf16_bits_to_float(X)


def test_training_gradient_matches_cpu_oracle():
    sim, _, _ = _collecting_sim()
    X, t = sim.ml_samples()
    assert len(t) > 2000
    rng = np.random.default_rng(11)
    w = (rng.normal(size=mlp.NPARAM) * 0.15).astype(np.float32)
    sim.ml_set_weights(w)
    rows = 1500
    loss, g = sim.ml_grad(100, rows)
    L, G = mlp.loss_and_grad(w, _features(X[100:100 + rows]), t[100:100 + rows])
    assert abs(loss - L) <= 1e-5 * max(1.0, L)
    assert np.linalg.norm(g - G) <= GRAD_TOL * np.linalg.norm(G)
    sim.close()


def test_tensor_core_inference_matches_bf16_emulation():
    sim, _, _ = _collecting_sim(steps=2)
    X, t = sim.ml_samples()
    rng = np.random.default_rng(12)
    w = (rng.normal(size=mlp.NPARAM) * 0.15).astype(np.float32)
    sim.ml_set_weights(w)
    rows = min(len(t), 4000) - 7        # not a multiple of the 16-row tile
    y = sim.ml_predict_samples(0, rows)
    ref = mlp.infer_bf16(w, _features(X[:rows]))
    assert np.linalg.norm(y - ref) <= INFER_TOL * np.linalg.norm(ref)
    sim.close()


def test_trained_warm_start_lowers_the_start_residual():
    sim, P, q = _collecting_sim(steps=10, every=1)
    loss = sim.ml_train(epochs=40, batch=1024, lr=2e-3, seed=5)
    X, t = sim.ml_samples()
    assert loss < 0.9 * float(np.mean(t.astype(np.float64) ** 2))   # better than predicting zero change
    w = sim.ml_get_weights()
    state, _, _ = sim.download()
    sim.close()
    its, fields = {}, {}
    for name, mode in (("plain", layout.PPE_MIXED_IR), ("learned", layout.PPE_LEARNED)):
        r = q.copy()
        r.ppe_mode = mode
        s2 = abi.Simulation(r, precision=layout.PREC_MIXED)
        s2.upload(state)
        if mode == layout.PPE_LEARNED:
            s2.ml_set_weights(w)
        total, init = 0, []
        for _ in range(5):
            st = s2.step(1)
            assert st.status == 0 and st.rel_residual <= 1e-6
            total += st.iterations
            init.append(st.initial_residual)
        its[name] = total
        its[name + "_initial_residual"] = float(np.mean(init))
        fields[name], _, _ = s2.download()
        s2.close()
    print("warm start", its)
    assert its["learned_initial_residual"] < 0.95 * its["plain_initial_residual"], its
    for f in ("ux", "uy", "uz"):
        a, b = fields["learned"][f].astype(np.float64), fields["plain"][f].astype(np.float64)
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max(), f
